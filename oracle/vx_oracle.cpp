/*
 * vx_oracle.cpp - CPU oracle: restatement of the reference's octree rebuild,
 * ESVO castRay, brick DDA and DXT1 colour codec.
 *
 * TEST INFRASTRUCTURE ONLY (see vx_oracle.h).  Nothing in the product links
 * this file.  Every function cites the reference file:line it restates; paths
 * are relative to the reference project's VIXEN/ directory.
 *
 * Substitutions (the reference's dependencies glm and gaia-ecs are not
 * installed here; oracle/ref_shim/ compiles the reference itself against
 * stand-ins for them, and tests/test_ref_pin.py holds this file to it):
 *  (1) glm -> V3 below, with glm's operation order: dot = (x*x + y*y) + z*z,
 *      normalize = v * (1 / sqrt(dot)), min(x,y) = (y < x) ? y : x,
 *      max(x,y) = (x < y) ? y : x, clamp = min(max(x, lo), hi).
 *  (2) gaia-ecs entity lookups -> a key set (or a dense bit grid) of occupied
 *      integer voxel positions.  A voxel counts as occupied when it exists
 *      (the reference DDA additionally requires a Density component > 0,
 *      GaiaVoxelWorld density test at SVOBrickDDA.cpp:462-468; every voxel of
 *      the ported tests carries Density{1}).
 *  (3) unordered_map brick lookups -> the same maps, exported as dense arrays.
 *  (4) ChildDescriptor::childPointer is 15 bits in the reference
 *      (SVOTypes.h:38) and is assigned without a far pointer
 *      (SVORebuild.cpp:584); here it is 32 bits, identical whenever the
 *      descriptor count is below 32768 (vxo_max_child_pointer reports it).
 *  (5) static_cast<int>(float) outside the int range is undefined in C++;
 *      x86-64 (cvttss2si) returns INT_MIN.  f2i() pins that behaviour.
 * Built with -O2 -ffp-contract=off -fno-fast-math so that every float
 * operation is a single IEEE-754 binary32 operation in source order.
 */
#include "vx_oracle.h"

#include <algorithm>
#include <array>
#include <bit>
#include <climits>
#include <cmath>
#include <cstring>
#include <limits>
#include <queue>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace {

// ---------------------------------------------------------------------------
// glm stand-ins (substitution 1)
// ---------------------------------------------------------------------------
struct V3 {
    float x, y, z;
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
};
struct I3 { int x, y, z; };

inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline V3 operator/(V3 a, V3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
inline V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline V3 splat(float s) { return {s, s, s}; }

inline float gmin(float x, float y) { return (y < x) ? y : x; }
inline float gmax(float x, float y) { return (x < y) ? y : x; }
inline int imin(int x, int y) { return (y < x) ? y : x; }
inline int imax(int x, int y) { return (x < y) ? y : x; }
inline V3 vmin(V3 a, V3 b) { return {gmin(a.x, b.x), gmin(a.y, b.y), gmin(a.z, b.z)}; }
inline V3 vmax(V3 a, V3 b) { return {gmax(a.x, b.x), gmax(a.y, b.y), gmax(a.z, b.z)}; }
inline V3 vclamp(V3 v, V3 lo, V3 hi) { return vmin(vmax(v, lo), hi); }
inline I3 iclamp(I3 v, int lo, int hi) {
    return {imin(imax(v.x, lo), hi), imin(imax(v.y, lo), hi), imin(imax(v.z, lo), hi)};
}
inline float dot(V3 a, V3 b) { V3 t = a * b; return (t.x + t.y) + t.z; }
inline float length(V3 v) { return std::sqrt(dot(v, v)); }
inline V3 normalize(V3 v) { return v * (1.0f / std::sqrt(dot(v, v))); }
// std::min({a,b,c}) / std::max({a,b,c}) as min_element/max_element
inline float min3(float a, float b, float c) { return gmin(gmin(a, b), c); }
inline float max3(float a, float b, float c) { return gmax(gmax(a, b), c); }

// Substitution 5: x86-64 static_cast<int>(float).
inline int f2i(float f) {
    if (f >= -2147483648.0f && f < 2147483648.0f) return static_cast<int>(f);
    return INT_MIN;
}

constexpr int ESVO_MAX_SCALE = 22;   // LaineKarrasOctree.h:337
constexpr int MAX_STACK_DEPTH = 32;  // LaineKarrasOctree.h:340
constexpr uint32_t NONE = 0xFFFFFFFFu;

// Hit flag encoding shared with the product (vx.h).
constexpr uint32_t F_HIT = 1u;
constexpr uint32_t F_AXIS_SHIFT = 1;
constexpr uint32_t F_NEG = 1u << 3;
constexpr uint32_t F_METHOD_SHIFT = 4;
constexpr uint32_t F_ITER_CAP = 1u << 6;
constexpr uint32_t F_INVALID = 1u << 7;

// ---------------------------------------------------------------------------
// Morton code (Core/src/MortonEncoding.cpp:19-63, offset 2^20 per axis)
// ---------------------------------------------------------------------------
uint64_t expandBits(uint32_t v) {
    uint64_t x = v & 0x1FFFFF;
    x = (x | x << 32) & 0x1F00000000FFFFULL;
    x = (x | x << 16) & 0x1F0000FF0000FFULL;
    x = (x | x << 8) & 0x100F00F00F00F00FULL;
    x = (x | x << 4) & 0x10C30C30C30C30C3ULL;
    x = (x | x << 2) & 0x1249249249249249ULL;
    return x;
}
uint64_t mortonFromWorldPos(int x, int y, int z) {
    const int32_t offset = 1048576;  // MortonCode64::COORDINATE_OFFSET
    return expandBits(uint32_t(x + offset)) | (expandBits(uint32_t(y + offset)) << 1) |
           (expandBits(uint32_t(z + offset)) << 2);
}

inline uint64_t packKey(int x, int y, int z) {
    return (uint64_t(uint32_t(x + 1048576)) & 0x1FFFFF) |
           ((uint64_t(uint32_t(y + 1048576)) & 0x1FFFFF) << 21) |
           ((uint64_t(uint32_t(z + 1048576)) & 0x1FFFFF) << 42);
}

// mirrorMask (SVOTypes.h:343-364)
inline uint8_t mirrorMask(uint8_t mask, int octant_mask) {
    if (octant_mask == 7) return mask;
    uint8_t flipMask = (~octant_mask) & 7;
    uint8_t result = 0;
    for (int i = 0; i < 8; i++) {
        int mirroredIdx = i ^ flipMask;
        if (mask & (1 << i)) result |= (1 << mirroredIdx);
    }
    return result;
}
inline int mirroredToLocalOctant(int mirroredIdx, int octant_mask) {  // SVOTypes.h:380-383
    return mirroredIdx ^ (~octant_mask & 7);
}

}  // namespace

// ---------------------------------------------------------------------------
// Scene (Octree + OctreeBlock of SVOBuilder.h:44-150, with substitution 2)
// ---------------------------------------------------------------------------
struct Desc {
    uint32_t childPointer;
    uint8_t validMask, leafMask;
    uint32_t brickIndex;  // contourPointer / brick index field
};

struct vxo_scene {
    V3 worldMin{0, 0, 0}, worldMax{1, 1, 1};
    int maxLevels = 23, brickDepthLevels = 3;
    int bricksPerAxis = 1, brickSideLength = 8;
    std::vector<Desc> desc;
    std::vector<I3> brickGrid;  // brickViews[i] grid coordinate
    std::unordered_map<uint32_t, uint32_t> brickGridToBrickView;
    std::unordered_map<uint64_t, uint32_t> leafToBrickView;
    // occupancy (substitution 2)
    bool dense = false;
    std::unordered_set<uint64_t> keys;
    std::vector<uint64_t> bits;
    int R = 0;
    I3 qwm{0, 0, 0};  // VolumeGrid::quantize(worldMin) (VoxelComponents.h:373-379)

    bool occupied(int kx, int ky, int kz) const {
        if (dense) {
            if (kx < 0 || ky < 0 || kz < 0 || kx >= R || ky >= R || kz >= R) return false;
            size_t w = (size_t(kz) * R + ky) * (R / 64) + (kx >> 6);
            return (bits[w] >> (kx & 63)) & 1u;
        }
        return keys.count(packKey(kx, ky, kz)) != 0;
    }
    // EntityBrickView::getEntity in LocalGrid mode (GaiaVoxelWorld/src/EntityBrickView.cpp:109-133)
    bool brickVoxelOccupied(uint32_t view, int x, int y, int z, I3* key) const {
        const I3 g = brickGrid[view];
        I3 k{g.x * brickSideLength + x + qwm.x, g.y * brickSideLength + y + qwm.y,
             g.z * brickSideLength + z + qwm.z};
        if (key) *key = k;
        return occupied(k.x, k.y, k.z);
    }
    int64_t getBrickViewByGrid(int bx, int by, int bz) const {  // SVOBuilder.h:107-116
        uint32_t key = uint32_t(bx) | (uint32_t(by) << 10) | (uint32_t(bz) << 20);
        auto it = brickGridToBrickView.find(key);
        if (it != brickGridToBrickView.end() && it->second < brickGrid.size()) return it->second;
        return -1;
    }
    int64_t getBrickView(size_t parentDescriptorIndex, int octant) const {  // SVOBuilder.h:96-104
        uint64_t key = (uint64_t(parentDescriptorIndex) << 3) | uint64_t(octant);
        auto it = leafToBrickView.find(key);
        if (it != leafToBrickView.end() && it->second < brickGrid.size()) return it->second;
        return -1;
    }
};

namespace {

// splitmix64 finaliser: a well-spread 64-bit hash of a packed key.
inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

void setErr(char* err, int errlen, const std::string& m) {
    if (err && errlen > 0) {
        std::strncpy(err, m.c_str(), size_t(errlen) - 1);
        err[errlen - 1] = 0;
    }
}

// ---------------------------------------------------------------------------
// LaineKarrasOctree::rebuild (SVO/src/SVORebuild.cpp:228-607), hierarchy part.
// `brickKeys` lists the populated brick grid coordinates (the binning result
// of :286-356); occupancy is already stored in the scene.
// ---------------------------------------------------------------------------
bool rebuildHierarchy(vxo_scene& s, const std::vector<I3>& populated, std::string& err) {
    const int brickDepth = s.brickDepthLevels;
    const int bricksPerAxis = s.bricksPerAxis;

    struct BrickInfo { I3 gridCoord; uint64_t mortonCode; };
    std::vector<BrickInfo> populatedBricks;
    populatedBricks.reserve(populated.size());
    for (const I3& g : populated) {
        // MortonCode64::fromWorldPos(localGridOrigin) (:346-347)
        populatedBricks.push_back({g, mortonFromWorldPos(g.x * s.brickSideLength,
                                                         g.y * s.brickSideLength,
                                                         g.z * s.brickSideLength)});
    }
    s.desc.clear();
    s.brickGrid.clear();
    s.brickGridToBrickView.clear();
    s.leafToBrickView.clear();
    if (populatedBricks.empty()) return true;  // :358-361 (empty octree)

    // Morton sort (:368-371); codes are unique per brick.
    std::sort(populatedBricks.begin(), populatedBricks.end(),
              [](const BrickInfo& a, const BrickInfo& b) { return a.mortonCode < b.mortonCode; });

    struct NodeKey {
        int depth; I3 coord;
        bool operator==(const NodeKey& o) const {
            return depth == o.depth && coord.x == o.coord.x && coord.y == o.coord.y && coord.z == o.coord.z;
        }
    };
    // The maps below only change the order in which nodes enter
    // tempDescriptors, which the BFS re-ordering removes; a mixing hash
    // replaces the reference's xor of shifted coordinates (which puts most
    // keys of a large scene into a few thousand buckets) without changing
    // any output.
    struct NodeKeyHash {
        size_t operator()(const NodeKey& k) const {
            return size_t(mix64(uint64_t(uint32_t(k.depth)) << 60 ^ uint64_t(uint32_t(k.coord.x)) ^
                                uint64_t(uint32_t(k.coord.y)) << 20 ^ uint64_t(uint32_t(k.coord.z)) << 40));
        }
    };
    std::unordered_map<NodeKey, uint32_t, NodeKeyHash> nodeToDescriptorIndex;
    std::vector<Desc> tempDescriptors;
    std::unordered_map<uint32_t, std::array<uint32_t, 8>> childMapping;

    // Brick-level nodes (:418-443)
    for (const auto& brick : populatedBricks) {
        NodeKey key{brickDepth, brick.gridCoord};
        uint32_t descriptorIndex = uint32_t(tempDescriptors.size());
        uint32_t brickViewIndex = uint32_t(s.brickGrid.size());
        nodeToDescriptorIndex[key] = descriptorIndex;
        uint32_t gridKey = uint32_t(brick.gridCoord.x) | (uint32_t(brick.gridCoord.y) << 10) |
                           (uint32_t(brick.gridCoord.z) << 20);
        s.brickGridToBrickView[gridKey] = brickViewIndex;
        Desc d{};
        d.validMask = 0xFF;
        d.leafMask = 0xFF;
        d.childPointer = 0;
        d.brickIndex = brickViewIndex & 0xFFFFFFu;  // setBrickIndex (SVOTypes.h:106-109)
        tempDescriptors.push_back(d);
        s.brickGrid.push_back(brick.gridCoord);
    }

    // Parent levels bottom-up (:446-518)
    for (int currentDepth = brickDepth + 1; currentDepth <= s.maxLevels; ++currentDepth) {
        struct IH {
            size_t operator()(const I3& v) const {
                return size_t(mix64(uint64_t(uint32_t(v.x)) ^ uint64_t(uint32_t(v.y)) << 21 ^
                                    uint64_t(uint32_t(v.z)) << 42));
            }
        };
        struct IE {
            bool operator()(const I3& a, const I3& b) const { return a.x == b.x && a.y == b.y && a.z == b.z; }
        };
        std::unordered_map<I3, std::vector<std::pair<int, uint32_t>>, IH, IE> parentToChildren;
        int childDepth = currentDepth - 1;
        for (const auto& [key, descriptorIndex] : nodeToDescriptorIndex) {
            if (key.depth != childDepth) continue;
            I3 parentCoord{key.coord.x / 2, key.coord.y / 2, key.coord.z / 2};
            int octant = (key.coord.x % 2) + ((key.coord.y % 2) << 1) + ((key.coord.z % 2) << 2);
            parentToChildren[parentCoord].push_back({octant, descriptorIndex});
        }
        if (parentToChildren.empty()) break;
        bool isRootLevel = (parentToChildren.size() == 1 && parentToChildren.count(I3{0, 0, 0}) == 1);
        for (const auto& [parentCoord, children] : parentToChildren) {
            uint32_t parentDescriptorIndex = uint32_t(tempDescriptors.size());
            nodeToDescriptorIndex[NodeKey{currentDepth, parentCoord}] = parentDescriptorIndex;
            uint8_t validMask = 0, leafMask = 0;
            std::array<uint32_t, 8> childIndices;
            childIndices.fill(UINT32_MAX);
            for (const auto& [octant, childIndex] : children) {
                validMask |= uint8_t(1 << octant);
                childIndices[octant] = childIndex;
                if (childDepth == brickDepth) leafMask |= uint8_t(1 << octant);
            }
            childMapping[parentDescriptorIndex] = childIndices;
            if (bricksPerAxis == 1 && children.size() == 1) {  // :496-502
                validMask = 0xFF;
                leafMask = 0xFF;
                childIndices.fill(children[0].second);
                childMapping[parentDescriptorIndex] = childIndices;
            }
            Desc pd{};
            pd.validMask = validMask;
            pd.leafMask = leafMask;
            pd.childPointer = 0;
            pd.brickIndex = 0;  // contourPointer = 0 (:509)
            tempDescriptors.push_back(pd);
        }
        if (isRootLevel) break;
    }

    // Root = descriptor of greatest depth (:526-534).  When several nodes share
    // the greatest depth the reference's choice depends on unordered_map
    // iteration order; such scenes are rejected.
    uint32_t rootOldIndex = UINT32_MAX;
    int rootDepth = -1, atRootDepth = 0;
    for (const auto& [key, index] : nodeToDescriptorIndex) {
        if (key.depth > rootDepth) { rootDepth = key.depth; rootOldIndex = index; atRootDepth = 1; }
        else if (key.depth == rootDepth) { ++atRootDepth; }
    }
    if (rootOldIndex == UINT32_MAX) return true;
    if (atRootDepth != 1) {
        err = "octree has several nodes at the top level (maxLevels too small for the bounds)";
        return false;
    }

    // BFS re-ordering (:540-598)
    struct NodeInfo { uint32_t oldIndex, newIndex; };
    std::queue<NodeInfo> bfsQueue;
    std::unordered_map<uint32_t, uint32_t> oldToNewIndex;
    std::vector<Desc>& finalDescriptors = s.desc;
    bfsQueue.push({rootOldIndex, 0});
    oldToNewIndex[rootOldIndex] = 0;
    finalDescriptors.push_back(tempDescriptors[rootOldIndex]);
    while (!bfsQueue.empty()) {
        NodeInfo current = bfsQueue.front();
        bfsQueue.pop();
        const Desc& desc = tempDescriptors[current.oldIndex];
        auto it = childMapping.find(current.oldIndex);
        if (it == childMapping.end()) continue;
        std::vector<uint32_t> nonLeafChildren, leafChildren;
        for (int octant = 0; octant < 8; ++octant) {
            if (!(desc.validMask & (1 << octant))) continue;
            uint32_t childOldIndex = it->second[octant];
            if (childOldIndex == UINT32_MAX) continue;
            if (desc.leafMask & (1 << octant)) {
                leafChildren.push_back(childOldIndex);
                uint64_t key = (uint64_t(current.newIndex) << 3) | uint64_t(octant);
                s.leafToBrickView[key] = tempDescriptors[childOldIndex].brickIndex;
            } else {
                nonLeafChildren.push_back(childOldIndex);
            }
        }
        std::vector<uint32_t> allChildren = nonLeafChildren;
        allChildren.insert(allChildren.end(), leafChildren.begin(), leafChildren.end());
        if (!allChildren.empty()) {
            uint32_t firstChildIndex = uint32_t(finalDescriptors.size());
            finalDescriptors[current.newIndex].childPointer = firstChildIndex;  // substitution 4
            for (uint32_t oldChildIndex : allChildren) {
                uint32_t newChildIndex = uint32_t(finalDescriptors.size());
                oldToNewIndex[oldChildIndex] = newChildIndex;
                finalDescriptors.push_back(tempDescriptors[oldChildIndex]);
            }
            for (uint32_t oldChildIndex : nonLeafChildren)
                bfsQueue.push({oldChildIndex, oldToNewIndex[oldChildIndex]});
        }
    }
    return true;
}

void initBounds(vxo_scene& s, V3 wmin, V3 wmax, int maxLevels, int brickDepth) {
    s.worldMin = wmin;
    s.worldMax = wmax;
    s.maxLevels = maxLevels;
    s.brickDepthLevels = brickDepth;
    s.brickSideLength = 1 << brickDepth;
    V3 worldSize = wmax - wmin;
    int voxelsPerAxis = f2i(worldSize.x);  // :261
    s.bricksPerAxis = (voxelsPerAxis + s.brickSideLength - 1) / s.brickSideLength;  // :262
    s.qwm = I3{f2i(std::floor(wmin.x)), f2i(std::floor(wmin.y)), f2i(std::floor(wmin.z))};
}

// ---------------------------------------------------------------------------
// Traversal types (LaineKarrasOctree.h:229-290, 346-370)
// ---------------------------------------------------------------------------
struct State {
    uint32_t parent = 0;
    uint64_t child_descriptor = 0;
    int idx = 0;
    int scale = 0;
    float scale_exp2 = 0.5f;
    V3 pos{1.0f, 1.0f, 1.0f};
    float t_min = 0.0f, t_max = 1.0f, h = 0.0f;
    float tx_center = 0.0f, ty_center = 0.0f, tz_center = 0.0f;
    uint8_t mirroredValidMask = 0, mirroredLeafMask = 0;
    int iter = 0;
};
struct Coef {
    float tx_coef = 0, ty_coef = 0, tz_coef = 0, tx_bias = 0, ty_bias = 0, tz_bias = 0;
    int octant_mask = 7;
    V3 rayDir{0, 0, 0}, normOrigin{1, 1, 1};
};
struct CastStack {
    uint32_t nodes[MAX_STACK_DEPTH];
    float tMax[MAX_STACK_DEPTH];
    void push(int scale, uint32_t node, float t) {
        if (scale >= 0 && scale < MAX_STACK_DEPTH) { nodes[scale] = node; tMax[scale] = t; }
    }
    uint32_t getNode(int scale) const {
        return (scale >= 0 && scale < MAX_STACK_DEPTH) ? nodes[scale] : NONE;
    }
    float getTMax(int scale) const {
        return (scale >= 0 && scale < MAX_STACK_DEPTH) ? tMax[scale] : 0.0f;
    }
};
struct Hit {
    bool hit = false;
    float tMin = 0, tMax = 0;
    V3 hitPoint{0, 0, 0}, normal{0, 0, 0};
    int scale = 0;
    uint32_t brick = NONE, node = NONE, voxel = 0xFFFF;
    I3 key{0, 0, 0};
    uint32_t flags = 0;
};
struct Counters { uint32_t grid_reads = 0, dda_steps = 0, leaf_visits = 0; };

// SVOTraversal.cpp:104-112
bool isPointInsideAABB(V3 p, V3 bmin, V3 bmax) {
    return p.x >= bmin.x && p.x <= bmax.x && p.y >= bmin.y && p.y <= bmax.y && p.z >= bmin.z &&
           p.z <= bmax.z;
}
// SVOTraversal.cpp:117-149
bool intersectAABB(V3 o, V3 d, V3 bmin, V3 bmax, float& tMin, float& tMax) {
    const float epsilon = 1e-8f;
    V3 invDir;
    for (int i = 0; i < 3; ++i) {
        if (std::abs(d[i]) < epsilon) {
            if (o[i] < bmin[i] || o[i] > bmax[i]) return false;
            invDir[i] = (d[i] >= 0.0f) ? 1e20f : -1e20f;
        } else {
            invDir[i] = 1.0f / d[i];
        }
    }
    V3 t0 = (bmin - o) * invDir;
    V3 t1 = (bmax - o) * invDir;
    V3 tNear = vmin(t0, t1);
    V3 tFar = vmax(t0, t1);
    tMin = max3(tNear.x, tNear.y, tNear.z);
    tMax = min3(tFar.x, tFar.y, tFar.z);
    return tMin <= tMax && tMax >= 0.0f;
}
// SVOTraversal.cpp:699-728
Coef computeRayCoefficients(V3 rayDir, V3 normOrigin) {
    Coef c;
    c.rayDir = rayDir;
    c.normOrigin = normOrigin;
    constexpr float epsilon = 1e-5f;
    V3 safe = rayDir;
    if (std::abs(safe.x) < epsilon) safe.x = std::copysignf(epsilon, safe.x);
    if (std::abs(safe.y) < epsilon) safe.y = std::copysignf(epsilon, safe.y);
    if (std::abs(safe.z) < epsilon) safe.z = std::copysignf(epsilon, safe.z);
    c.tx_coef = 1.0f / -std::abs(safe.x);
    c.ty_coef = 1.0f / -std::abs(safe.y);
    c.tz_coef = 1.0f / -std::abs(safe.z);
    c.tx_bias = c.tx_coef * normOrigin.x;
    c.ty_bias = c.ty_coef * normOrigin.y;
    c.tz_bias = c.tz_coef * normOrigin.z;
    c.octant_mask = 7;
    if (rayDir.x > 0.0f) { c.octant_mask ^= 1; c.tx_bias = 3.0f * c.tx_coef - c.tx_bias; }
    if (rayDir.y > 0.0f) { c.octant_mask ^= 2; c.ty_bias = 3.0f * c.ty_coef - c.ty_bias; }
    if (rayDir.z > 0.0f) { c.octant_mask ^= 4; c.tz_bias = 3.0f * c.tz_coef - c.tz_bias; }
    return c;
}
// SVOTraversal.cpp:730-766
void selectInitialOctant(State& st, const Coef& c) {
    constexpr float axis_epsilon = 1e-5f;
    constexpr float boundary_epsilon = 0.01f;
    bool usePos = (st.t_min < boundary_epsilon);
    float mx = (c.octant_mask & 1) ? c.normOrigin.x : (3.0f - c.normOrigin.x);
    float my = (c.octant_mask & 2) ? c.normOrigin.y : (3.0f - c.normOrigin.y);
    float mz = (c.octant_mask & 4) ? c.normOrigin.z : (3.0f - c.normOrigin.z);
    if (std::abs(c.rayDir.x) < axis_epsilon || usePos) {
        if (mx >= 1.5f) { st.idx |= 1; st.pos.x = 1.5f; }
    } else {
        if (1.5f * c.tx_coef - c.tx_bias > st.t_min) { st.idx ^= 1; st.pos.x = 1.5f; }
    }
    if (std::abs(c.rayDir.y) < axis_epsilon || usePos) {
        if (my >= 1.5f) { st.idx |= 2; st.pos.y = 1.5f; }
    } else {
        if (1.5f * c.ty_coef - c.ty_bias > st.t_min) { st.idx ^= 2; st.pos.y = 1.5f; }
    }
    if (std::abs(c.rayDir.z) < axis_epsilon || usePos) {
        if (mz >= 1.5f) { st.idx |= 4; st.pos.z = 1.5f; }
    } else {
        if (1.5f * c.tz_coef - c.tz_bias > st.t_min) { st.idx ^= 4; st.pos.z = 1.5f; }
    }
}
// SVOTraversal.cpp:768-784
float computeCorrectedTcMax(float tx, float ty, float tz, V3 rayDir, float t_max) {
    constexpr float corner_threshold = 1000.0f;
    constexpr float dir_epsilon = 1e-5f;
    bool ux = std::abs(rayDir.x) >= dir_epsilon;
    bool uy = std::abs(rayDir.y) >= dir_epsilon;
    bool uz = std::abs(rayDir.z) >= dir_epsilon;
    float txv = (ux && std::abs(tx) < corner_threshold) ? tx : t_max;
    float tyv = (uy && std::abs(ty) < corner_threshold) ? ty : t_max;
    float tzv = (uz && std::abs(tz) < corner_threshold) ? tz : t_max;
    return min3(txv, tyv, tzv);
}
// SVOTraversal.cpp:786-794
inline void computeVoxelCorners(V3 pos, const Coef& c, float& tx, float& ty, float& tz) {
    tx = pos.x * c.tx_coef - c.tx_bias;
    ty = pos.y * c.ty_coef - c.ty_bias;
    tz = pos.z * c.tz_coef - c.tz_bias;
}

// LaineKarrasOctree::traverseBrickView (SVOBrickDDA.cpp:390-533)
bool traverseBrickView(const vxo_scene& s, uint32_t view, V3 brickWorldMin, float brickVoxelSize,
                       V3 rayOrigin, V3 rayDir, float tMin, float tMax, Hit& hit, Counters& cnt) {
    const int brickN = 1 << s.brickDepthLevels;
    const V3 entryPoint = rayOrigin + rayDir * tMin;
    const V3 localEntry = (entryPoint - brickWorldMin) / brickVoxelSize;
    I3 cur{f2i(std::floor(localEntry.x)), f2i(std::floor(localEntry.y)), f2i(std::floor(localEntry.z))};
    cur = iclamp(cur, 0, brickN - 1);
    int step[3];
    float tDelta[3], tNext[3];
    int curv[3] = {cur.x, cur.y, cur.z};
    constexpr float epsilon = 1e-8f;
    for (int axis = 0; axis < 3; ++axis) {
        if (std::abs(rayDir[axis]) < epsilon) {
            step[axis] = 0;
            tDelta[axis] = std::numeric_limits<float>::max();
            tNext[axis] = std::numeric_limits<float>::max();
        } else {
            step[axis] = (rayDir[axis] > 0.0f) ? 1 : -1;
            tDelta[axis] = brickVoxelSize / std::abs(rayDir[axis]);
            if (rayDir[axis] > 0.0f) {
                const float nextBoundaryWorld = brickWorldMin[axis] + float(curv[axis] + 1) * brickVoxelSize;
                const float dist = nextBoundaryWorld - entryPoint[axis];
                tNext[axis] = tMin + dist / rayDir[axis];
            } else {
                const float nextBoundaryWorld = brickWorldMin[axis] + float(curv[axis]) * brickVoxelSize;
                const float dist = entryPoint[axis] - nextBoundaryWorld;
                tNext[axis] = tMin + dist / std::abs(rayDir[axis]);
            }
        }
    }
    int maxSteps = brickN * 3;
    int stepCount = 0;
    while (stepCount < maxSteps) {
        ++stepCount;
        if (curv[0] < 0 || curv[0] >= brickN || curv[1] < 0 || curv[1] >= brickN || curv[2] < 0 ||
            curv[2] >= brickN)
            return false;
        ++cnt.dda_steps;
        I3 key;
        bool occ = s.brickVoxelOccupied(view, curv[0], curv[1], curv[2], &key);
        if (occ) {
            V3 vmin_{brickWorldMin.x + float(curv[0]) * brickVoxelSize,
                     brickWorldMin.y + float(curv[1]) * brickVoxelSize,
                     brickWorldMin.z + float(curv[2]) * brickVoxelSize};
            V3 vmax_ = vmin_ + splat(brickVoxelSize);
            V3 t0, t1;
            for (int i = 0; i < 3; i++) {
                if (std::abs(rayDir[i]) < 1e-8f) {
                    t0[i] = -std::numeric_limits<float>::infinity();
                    t1[i] = std::numeric_limits<float>::infinity();
                } else {
                    t0[i] = (vmin_[i] - rayOrigin[i]) / rayDir[i];
                    t1[i] = (vmax_[i] - rayOrigin[i]) / rayDir[i];
                }
            }
            V3 tNearHit = vmin(t0, t1);
            float hitT = gmax(gmax(tNearHit.x, tNearHit.y), tNearHit.z);
            hitT = gmax(hitT, 0.0f);
            int axis;
            if (tNearHit.x >= tNearHit.y && tNearHit.x >= tNearHit.z) axis = 0;
            else if (tNearHit.y >= tNearHit.z) axis = 1;
            else axis = 2;
            V3 n{0, 0, 0};
            n[axis] = rayDir[axis] > 0.0f ? -1.0f : 1.0f;
            hit.hit = true;
            hit.tMin = hitT;
            hit.tMax = hitT + brickVoxelSize;
            hit.hitPoint = rayOrigin + rayDir * hitT;
            hit.scale = s.maxLevels - 1;
            hit.normal = n;
            hit.voxel = uint32_t(curv[2] * 64 + curv[1] * 8 + curv[0]);
            hit.key = key;
            hit.flags |= F_HIT | (uint32_t(axis) << F_AXIS_SHIFT) | (rayDir[axis] > 0.0f ? F_NEG : 0u);
            return true;
        }
        if (tNext[0] < tNext[1] && tNext[0] < tNext[2]) {
            if (tNext[0] > tMax) return false;
            curv[0] += step[0];
            tNext[0] += tDelta[0];
        } else if (tNext[1] < tNext[2]) {
            if (tNext[1] > tMax) return false;
            curv[1] += step[1];
            tNext[1] += tDelta[1];
        } else {
            if (tNext[2] > tMax) return false;
            curv[2] += step[2];
            tNext[2] += tDelta[2];
        }
    }
    return false;
}

// traverseBrickAndReturnHit (SVOBrickDDA.cpp:187-225)
bool traverseBrickAndReturnHit(const vxo_scene& s, uint32_t view, V3 o, V3 d, float tEntry, Hit& hit,
                               Counters& cnt) {
    const float brickSideLength = float(1u << s.brickDepthLevels);
    constexpr float brickVoxelSize = 1.0f;
    const I3 g = s.brickGrid[view];
    V3 bmin{float(g.x * s.brickSideLength), float(g.y * s.brickSideLength), float(g.z * s.brickSideLength)};
    V3 bmax = bmin + splat(brickSideLength * brickVoxelSize);
    V3 invDir;
    for (int i = 0; i < 3; i++) {
        if (std::abs(d[i]) < 1e-8f) invDir[i] = (d[i] >= 0) ? 1e8f : -1e8f;
        else invDir[i] = 1.0f / d[i];
    }
    V3 t0 = (bmin - o) * invDir;
    V3 t1 = (bmax - o) * invDir;
    V3 tNear = vmin(t0, t1);
    V3 tFar = vmax(t0, t1);
    float brickTMin = gmax(gmax(tNear.x, tNear.y), tNear.z);
    float brickTMax = gmin(gmin(tFar.x, tFar.y), tFar.z);
    brickTMin = gmax(brickTMin, tEntry);
    return traverseBrickView(s, view, bmin, brickVoxelSize, o, d, brickTMin, brickTMax, hit, cnt);
}

// LaineKarrasOctree::handleLeafHit (SVOBrickDDA.cpp:65-181)
bool handleLeafHit(const vxo_scene& s, const State& st, const Coef& c, V3 origin, float tEntry, Hit& hit,
                   Counters& cnt) {
    ++cnt.leaf_visits;
    size_t parentDescriptorIndex = st.parent;
    V3 worldSize = s.worldMax - s.worldMin;
    int bricksPerAxis = s.bricksPerAxis;
    float brickSide = float(s.brickSideLength);
    constexpr float axis_epsilon = 1e-5f;
    V3 localPos = st.pos;
    float octantSize = st.scale_exp2;
    if ((c.octant_mask & 1) == 0) localPos.x = 3.0f - octantSize - localPos.x;
    if ((c.octant_mask & 2) == 0) localPos.y = 3.0f - octantSize - localPos.y;
    if ((c.octant_mask & 4) == 0) localPos.z = 3.0f - octantSize - localPos.z;
    V3 localNorm = localPos - splat(1.0f);
    float offset = 0.001f;
    V3 offsetDir{(c.rayDir.x > 0) ? offset : -offset, (c.rayDir.y > 0) ? offset : -offset,
                 (c.rayDir.z > 0) ? offset : -offset};
    V3 octantInside = localNorm + offsetDir;
    V3 rayPosWorld = origin + c.rayDir * gmax(tEntry, 0.0f);
    V3 rayPosLocal = (rayPosWorld - s.worldMin) / worldSize;
    rayPosLocal = vclamp(rayPosLocal, splat(0.001f), splat(0.999f));
    if (std::abs(c.rayDir.x) < axis_epsilon) octantInside.x = rayPosLocal.x;
    if (std::abs(c.rayDir.y) < axis_epsilon) octantInside.y = rayPosLocal.y;
    if (std::abs(c.rayDir.z) < axis_epsilon) octantInside.z = rayPosLocal.z;
    octantInside = vclamp(octantInside, splat(0.001f), splat(0.999f));

    int64_t bv = -1;
    uint32_t method = 0;
    // Method 1: ESVO state position
    V3 hitPosLocal = octantInside * worldSize;
    hitPosLocal = vclamp(hitPosLocal, splat(0.0f), worldSize - splat(0.001f));
    I3 bi{f2i(hitPosLocal.x / brickSide), f2i(hitPosLocal.y / brickSide), f2i(hitPosLocal.z / brickSide)};
    bi = iclamp(bi, 0, bricksPerAxis - 1);
    ++cnt.grid_reads;
    bv = s.getBrickViewByGrid(bi.x, bi.y, bi.z);
    if (bv >= 0) method = 1;
    // Method 2: ray entry position
    if (bv < 0) {
        V3 rayEntryWorld = origin + c.rayDir * gmax(tEntry, 0.0f);
        V3 rayEntryLocal = rayEntryWorld - s.worldMin;
        rayEntryLocal = rayEntryLocal + c.rayDir * 0.01f;
        rayEntryLocal = vclamp(rayEntryLocal, splat(0.0f), worldSize - splat(0.001f));
        bi = I3{f2i(rayEntryLocal.x / brickSide), f2i(rayEntryLocal.y / brickSide),
                f2i(rayEntryLocal.z / brickSide)};
        bi = iclamp(bi, 0, bricksPerAxis - 1);
        ++cnt.grid_reads;
        bv = s.getBrickViewByGrid(bi.x, bi.y, bi.z);
        if (bv >= 0) method = 2;
    }
    // Fallback 3: ESVO octant-based lookup
    if (bv < 0) {
        int localOctant = mirroredToLocalOctant(st.idx, c.octant_mask);
        bv = s.getBrickView(parentDescriptorIndex, localOctant);
        if (bv >= 0) method = 3;
    }
    if (bv < 0) return false;
    // worldToLocal = inverse(translate(worldMin)) (SVORebuild.cpp:248-255)
    V3 localRayOrigin = origin + (splat(0.0f) - s.worldMin);
    V3 localRayDir = c.rayDir;
    hit.flags |= method << F_METHOD_SHIFT;
    bool r = traverseBrickAndReturnHit(s, uint32_t(bv), localRayOrigin, localRayDir, tEntry, hit, cnt);
    if (r) {
        hit.hitPoint = hit.hitPoint + s.worldMin;
        hit.brick = uint32_t(bv);
        hit.node = uint32_t(parentDescriptorIndex);
    } else {
        hit.flags &= ~(3u << F_METHOD_SHIFT);
    }
    return r;
}

// LODParameters (SVO/include/SVOLOD.h:50-177): cone diameter at the origin and
// its growth per unit distance; LOD is on when rayDirSize > 0 (:156-158).
struct Lod { float rayOrigSize = 0.0f, rayDirSize = 0.0f; };

// LaineKarrasOctree::castRayImpl (SVOTraversal.cpp:516-691); lod == nullptr is
// castRay, otherwise castRayWithLOD (:198-232, termination :613-651).
Hit castRay(const vxo_scene& s, V3 origin, V3 direction, float tMin, float tMax, uint32_t& itersOut,
            Counters& cnt, const Lod* lod = nullptr) {
    Hit miss;
    itersOut = 0;
    // validateRayInput (:238-259)
    if (s.desc.empty()) { miss.flags |= F_INVALID; return miss; }
    V3 rayDir = normalize(direction);
    float rayLength = length(rayDir);
    if (rayLength < 1e-6f) { miss.flags |= F_INVALID; return miss; }
    if (std::isnan(origin.x) || std::isnan(origin.y) || std::isnan(origin.z) || std::isnan(rayDir.x) ||
        std::isnan(rayDir.y) || std::isnan(rayDir.z) || std::isinf(origin.x) || std::isinf(origin.y) ||
        std::isinf(origin.z) || std::isinf(rayDir.x) || std::isinf(rayDir.y) || std::isinf(rayDir.z)) {
        miss.flags |= F_INVALID;
        return miss;
    }
    bool rayStartsInside = isPointInsideAABB(origin, s.worldMin, s.worldMax);
    float tEntry, tExit;
    if (!intersectAABB(origin, rayDir, s.worldMin, s.worldMax, tEntry, tExit)) return miss;
    tEntry = gmax(tEntry, tMin);
    tExit = gmin(tExit, tMax);
    if (tEntry >= tExit || tExit < 0.0f) return miss;
    float tRayStart = rayStartsInside ? 0.0f : gmax(0.0f, tEntry);
    V3 rayEntryPoint = origin + rayDir * tRayStart;
    V3 worldSize = s.worldMax - s.worldMin;
    V3 normOrigin = (rayEntryPoint - s.worldMin) / worldSize + splat(1.0f);
    float worldRayLength = length(worldSize);  // :552
    Coef coef = computeRayCoefficients(rayDir, normOrigin);
    State st;
    if (rayStartsInside) {
        st.t_min = 0.0f;
        st.t_max = min3(coef.tx_coef - coef.tx_bias, coef.ty_coef - coef.ty_bias, coef.tz_coef - coef.tz_bias);
        st.t_max = gmin(st.t_max, 1.0f);
    } else {
        st.t_min = max3(2.0f * coef.tx_coef - coef.tx_bias, 2.0f * coef.ty_coef - coef.ty_bias,
                        2.0f * coef.tz_coef - coef.tz_bias);
        st.t_max = min3(coef.tx_coef - coef.tx_bias, coef.ty_coef - coef.ty_bias, coef.tz_coef - coef.tz_bias);
        st.t_min = gmax(st.t_min, 0.0f);
        st.t_max = gmin(st.t_max, 1.0f);
    }
    st.h = st.t_max;

    // initializeTraversalState (:261-280)
    CastStack stack;
    const int minScale = ESVO_MAX_SCALE - s.maxLevels + 1;
    for (int sc = minScale; sc <= ESVO_MAX_SCALE; sc++) stack.push(sc, 0, st.t_max);
    st.scale = ESVO_MAX_SCALE;
    st.parent = 0;
    st.child_descriptor = 0;
    st.idx = 0;
    st.pos = V3{1.0f, 1.0f, 1.0f};
    st.scale_exp2 = 0.5f;
    selectInitialOctant(st, coef);

    const int maxIter = 500;
    const int nodeCount = int(s.desc.size());
    const int brickUserScale = s.maxLevels - s.brickDepthLevels;
    constexpr float dir_epsilon = 1e-5f;
    while (st.scale >= minScale && st.scale <= ESVO_MAX_SCALE && st.iter < maxIter) {
        ++st.iter;
        // fetchChildDescriptor (:282-293)
        if (st.child_descriptor == 0) {
            const Desc& p = s.desc[st.parent];
            st.mirroredValidMask = mirrorMask(p.validMask, coef.octant_mask);
            st.mirroredLeafMask = mirrorMask(p.leafMask, coef.octant_mask);
            uint32_t nonLeafMask = ~uint32_t(st.mirroredLeafMask) & 0xFF;
            st.child_descriptor = nonLeafMask | (uint64_t(st.mirroredValidMask) << 8) |
                                  (uint64_t(p.childPointer) << 16);
        }
        // checkChildValidity (:295-326)
        bool isLeaf;
        float tv_max = 0.0f;
        bool shouldProcess;
        {
            bool child_valid = (st.mirroredValidMask & (1u << st.idx)) != 0;
            isLeaf = (st.mirroredLeafMask & (1u << st.idx)) != 0;
            int currentUserScale = st.scale - (ESVO_MAX_SCALE - s.maxLevels + 1);
            if (currentUserScale == brickUserScale && child_valid) isLeaf = true;
            if (!child_valid || st.t_min > st.t_max) {
                shouldProcess = false;
            } else {
                float tx, ty, tz;
                computeVoxelCorners(st.pos, coef, tx, ty, tz);
                float tcc = computeCorrectedTcMax(tx, ty, tz, coef.rayDir, st.t_max);
                tv_max = gmin(st.t_max, tcc);
                float half = st.scale_exp2 * 0.5f;
                st.tx_center = half * coef.tx_coef + tx;
                st.ty_center = half * coef.ty_coef + ty;
                st.tz_center = half * coef.tz_coef + tz;
                shouldProcess = st.t_min <= tv_max;
            }
        }
        bool skipToAdvance = false;
        if (shouldProcess) {
            // Screen-space LOD termination (:613-651): world distance of the
            // cell entry, esvoScaleToWorldSize (SVOLOD.h:189-195) and
            // shouldTerminate (SVOLOD.h:129-146).
            if (lod != nullptr && lod->rayDirSize > 0.0f) {
                float worldDistance = tRayStart + st.t_min * worldRayLength;
                float worldVoxelSize = std::ldexp(1.0f, st.scale - ESVO_MAX_SCALE - 1) * worldSize.x;
                float projected = worldDistance * lod->rayDirSize + lod->rayOrigSize;
                if (projected >= worldVoxelSize) {
                    Hit h;
                    h.hit = true;
                    h.hitPoint = origin + rayDir * worldDistance;
                    h.normal = V3{0.0f, 1.0f, 0.0f};
                    h.tMin = worldDistance;
                    h.tMax = worldDistance + worldVoxelSize;
                    h.scale = st.scale - (ESVO_MAX_SCALE - s.maxLevels + 1);  // esvoToUserScale
                    h.node = st.parent;  // no entity: the cut cell is child idx of this descriptor
                    h.flags = F_HIT | (1u << 1);
                    itersOut = uint32_t(st.iter);
                    return h;
                }
            }
            if (isLeaf) {
                Hit h;
                if (handleLeafHit(s, st, coef, origin, tEntry, h, cnt)) {
                    itersOut = uint32_t(st.iter);
                    return h;
                }
                st.t_min = tv_max;
                skipToAdvance = true;
            }
            if (!skipToAdvance) {
                // executePushPhase (:328-378)
                float tx, ty, tz;
                computeVoxelCorners(st.pos, coef, tx, ty, tz);
                float tc_max = min3(tx, ty, tz);
                if (tc_max < st.h) stack.push(st.scale, st.parent, st.t_max);
                st.h = tc_max;
                int worldIdx = mirroredToLocalOctant(st.idx, coef.octant_mask);
                const Desc& p = s.desc[st.parent];
                uint8_t nonLeafMask = uint8_t(~p.leafMask & p.validMask);
                uint32_t mask_before_child = (1u << worldIdx) - 1;
                uint32_t child_offset = std::popcount(uint32_t(nonLeafMask) & mask_before_child);
                uint32_t child_index = p.childPointer + child_offset;
                if (child_index >= uint32_t(nodeCount)) continue;
                st.parent = child_index;
                st.idx = 0;
                st.scale--;
                float half = st.scale_exp2 * 0.5f;
                st.scale_exp2 = half;
                if (st.tx_center > st.t_min) { st.idx ^= 1; st.pos.x += st.scale_exp2; }
                if (st.ty_center > st.t_min) { st.idx ^= 2; st.pos.y += st.scale_exp2; }
                if (st.tz_center > st.t_min) { st.idx ^= 4; st.pos.z += st.scale_exp2; }
                st.t_max = tv_max;
                st.child_descriptor = 0;
                continue;
            }
        }
        // executeAdvancePhase (:380-416)
        bool popNeeded;
        {
            float tx, ty, tz;
            computeVoxelCorners(st.pos, coef, tx, ty, tz);
            bool csx = std::abs(coef.rayDir.x) >= dir_epsilon;
            bool csy = std::abs(coef.rayDir.y) >= dir_epsilon;
            bool csz = std::abs(coef.rayDir.z) >= dir_epsilon;
            float tcc = computeCorrectedTcMax(tx, ty, tz, coef.rayDir, st.t_max);
            if (tcc == std::numeric_limits<float>::max()) {
                const float L = -std::numeric_limits<float>::max();
                tcc = max3(csx ? tx : L, csy ? ty : L, csz ? tz : L);
            }
            int step_mask = 0;
            if (csx && tx <= tcc) { step_mask ^= 1; st.pos.x -= st.scale_exp2; }
            if (csy && ty <= tcc) { step_mask ^= 2; st.pos.y -= st.scale_exp2; }
            if (csz && tz <= tcc) { step_mask ^= 4; st.pos.z -= st.scale_exp2; }
            st.t_min = gmax(tcc, 0.0f);
            st.idx ^= step_mask;
            popNeeded = (st.idx & step_mask) != 0;
        }
        if (popNeeded) {
            // step mask recomputed at the new position (:672-681)
            float tx, ty, tz;
            computeVoxelCorners(st.pos, coef, tx, ty, tz);
            float tcc = computeCorrectedTcMax(tx, ty, tz, coef.rayDir, st.t_max);
            int step_mask = 0;
            if (std::abs(coef.rayDir.x) >= dir_epsilon && tx <= tcc) step_mask ^= 1;
            if (std::abs(coef.rayDir.y) >= dir_epsilon && ty <= tcc) step_mask ^= 2;
            if (std::abs(coef.rayDir.z) >= dir_epsilon && tz <= tcc) step_mask ^= 4;
            // executePopPhase (:418-510)
            bool exitOctree = false;
            if (st.scale == ESVO_MAX_SCALE) {
                if (st.t_min > st.t_max || st.pos.x < 1.0f || st.pos.x >= 2.0f || st.pos.y < 1.0f ||
                    st.pos.y >= 2.0f || st.pos.z < 1.0f || st.pos.z >= 2.0f) {
                    exitOctree = true;
                } else {
                    st.child_descriptor = 0;
                }
            } else {
                const int MAX_RES = 1 << ESVO_MAX_SCALE;
                auto floatToInt = [](float f) -> uint32_t {
                    float clamped = std::max(0.0f, std::min(f, 1.0f));
                    return static_cast<uint32_t>(std::max(0.0f, std::min(clamped * float(1 << ESVO_MAX_SCALE),
                                                                         float((1 << ESVO_MAX_SCALE) - 1))));
                };
                uint32_t px = floatToInt(std::max(0.0f, st.pos.x - 1.0f));
                uint32_t py = floatToInt(std::max(0.0f, st.pos.y - 1.0f));
                uint32_t pz = floatToInt(std::max(0.0f, st.pos.z - 1.0f));
                uint32_t nx = (step_mask & 1) ? floatToInt(std::max(0.0f, st.pos.x + st.scale_exp2 - 1.0f)) : px;
                uint32_t ny = (step_mask & 2) ? floatToInt(std::max(0.0f, st.pos.y + st.scale_exp2 - 1.0f)) : py;
                uint32_t nz = (step_mask & 4) ? floatToInt(std::max(0.0f, st.pos.z + st.scale_exp2 - 1.0f)) : pz;
                uint32_t differing = 0;
                if (step_mask & 1) differing |= (px ^ nx);
                if (step_mask & 2) differing |= (py ^ ny);
                if (step_mask & 4) differing |= (pz ^ nz);
                if (differing == 0) {
                    exitOctree = true;
                } else {
                    int highest_bit = 31 - std::countl_zero(differing);
                    st.scale = highest_bit;
                    if (st.scale < minScale || st.scale > ESVO_MAX_SCALE) {
                        exitOctree = true;
                    } else {
                        int exp_val = st.scale - ESVO_MAX_SCALE + 127;
                        st.scale_exp2 = std::bit_cast<float>(uint32_t(exp_val << 23));
                        st.parent = stack.getNode(st.scale);
                        st.t_max = stack.getTMax(st.scale);
                        int shift_amount = ESVO_MAX_SCALE - st.scale;
                        uint32_t mask = ~((1u << shift_amount) - 1);
                        px &= mask; py &= mask; pz &= mask;
                        st.pos.x = 1.0f + float(px) / float(MAX_RES);
                        st.pos.y = 1.0f + float(py) / float(MAX_RES);
                        st.pos.z = 1.0f + float(pz) / float(MAX_RES);
                        int idx_shift = ESVO_MAX_SCALE - st.scale - 1;
                        if (idx_shift < 0 || idx_shift >= 32) st.idx = 0;
                        else st.idx = int(((px >> idx_shift) & 1) | (((py >> idx_shift) & 1) << 1) |
                                          (((pz >> idx_shift) & 1) << 2));
                        st.h = 0.0f;
                        st.child_descriptor = 0;
                    }
                }
            }
            if (exitOctree) break;
        }
    }
    itersOut = uint32_t(st.iter);
    if (st.iter >= maxIter) miss.flags |= F_ITER_CAP;
    return miss;
}

}  // namespace

// ---------------------------------------------------------------------------
// C interface
// ---------------------------------------------------------------------------
extern "C" {

vxo_scene* vxo_build_from_keys(const int32_t* keys_xyz, uint64_t n, const float wmin[3], const float wmax[3],
                               int max_levels, int brick_depth, char* err, int errlen) {
    if (max_levels < 1 || max_levels > 23 || brick_depth != 3) {
        setErr(err, errlen, "max_levels must be in [1,23] and brick_depth must be 3");
        return nullptr;
    }
    auto* s = new vxo_scene();
    initBounds(*s, V3{wmin[0], wmin[1], wmin[2]}, V3{wmax[0], wmax[1], wmax[2]}, max_levels, brick_depth);
    if (s->bricksPerAxis < 1 || s->bricksPerAxis > 1024) {
        setErr(err, errlen, "bricks per axis out of range");
        delete s;
        return nullptr;
    }
    s->dense = false;
    s->keys.reserve(size_t(n) * 2);
    // Brick binning (SVORebuild.cpp:286-356): world integer position / 8, clamped.
    std::unordered_map<uint64_t, size_t> brickCounts;
    const int bs = s->brickSideLength, bpa = s->bricksPerAxis;
    for (uint64_t i = 0; i < n; ++i) {
        int x = keys_xyz[3 * i], y = keys_xyz[3 * i + 1], z = keys_xyz[3 * i + 2];
        s->keys.insert(packKey(x, y, z));
        int bx = std::clamp(x / bs, 0, bpa - 1);
        int by = std::clamp(y / bs, 0, bpa - 1);
        int bz = std::clamp(z / bs, 0, bpa - 1);
        brickCounts[uint64_t(bx) | (uint64_t(by) << 16) | (uint64_t(bz) << 32)]++;
    }
    std::vector<I3> populated;
    populated.reserve(brickCounts.size());
    for (const auto& kv : brickCounts)
        populated.push_back(I3{int(kv.first & 0xFFFF), int((kv.first >> 16) & 0xFFFF), int((kv.first >> 32) & 0xFFFF)});
    std::string e;
    if (!rebuildHierarchy(*s, populated, e)) {
        setErr(err, errlen, e);
        delete s;
        return nullptr;
    }
    return s;
}

vxo_scene* vxo_build_from_dense(const uint64_t* bits, int R, int max_levels, int brick_depth, char* err,
                                int errlen) {
    if (R < 64 || R % 64 != 0 || max_levels < 1 || max_levels > 23 || brick_depth != 3) {
        setErr(err, errlen, "R must be a positive multiple of 64, max_levels in [1,23], brick_depth 3");
        return nullptr;
    }
    auto* s = new vxo_scene();
    initBounds(*s, V3{0, 0, 0}, V3{float(R), float(R), float(R)}, max_levels, brick_depth);
    s->dense = true;
    s->R = R;
    const size_t words = size_t(R) * R * (R / 64);
    s->bits.assign(bits, bits + words);
    // Binning of every present voxel by position / 8: a brick is populated
    // when its 8^3 region holds a voxel.
    const int bpa = s->bricksPerAxis;
    std::vector<I3> populated;
    for (int bz = 0; bz < bpa; ++bz)
        for (int by = 0; by < bpa; ++by)
            for (int bx = 0; bx < bpa; ++bx) {
                bool any = false;
                for (int z = 0; z < 8 && !any; ++z)
                    for (int y = 0; y < 8 && !any; ++y) {
                        size_t w = (size_t(bz * 8 + z) * R + size_t(by * 8 + y)) * (R / 64) + (bx >> 3);
                        if ((s->bits[w] >> ((bx & 7) * 8)) & 0xFF) any = true;
                    }
                if (any) populated.push_back(I3{bx, by, bz});
            }
    std::string e;
    if (!rebuildHierarchy(*s, populated, e)) {
        setErr(err, errlen, e);
        delete s;
        return nullptr;
    }
    return s;
}

vxo_scene* vxo_build_from_descriptors(const uint32_t* nodes, const uint32_t* node_brick, uint32_t node_count,
                                      const float wmin[3], const float wmax[3], int max_levels,
                                      int brick_depth) {
    auto* s = new vxo_scene();
    initBounds(*s, V3{wmin[0], wmin[1], wmin[2]}, V3{wmax[0], wmax[1], wmax[2]}, max_levels, brick_depth);
    s->desc.resize(node_count);
    for (uint32_t i = 0; i < node_count; ++i) {
        s->desc[i].childPointer = nodes[2 * i];
        s->desc[i].validMask = uint8_t(nodes[2 * i + 1] & 0xFF);
        s->desc[i].leafMask = uint8_t((nodes[2 * i + 1] >> 8) & 0xFF);
        s->desc[i].brickIndex = node_brick ? node_brick[i] : 0;
    }
    return s;
}

void vxo_free(vxo_scene* s) { delete s; }
uint32_t vxo_node_count(const vxo_scene* s) { return uint32_t(s->desc.size()); }
uint32_t vxo_brick_count(const vxo_scene* s) { return uint32_t(s->brickGrid.size()); }
int32_t vxo_bricks_per_axis(const vxo_scene* s) { return s->bricksPerAxis; }
uint32_t vxo_max_child_pointer(const vxo_scene* s) {
    uint32_t m = 0;
    for (const auto& d : s->desc) m = std::max(m, d.childPointer);
    return m;
}

void vxo_export(const vxo_scene* s, uint32_t* nodes, uint32_t* node_brick, uint32_t* grid_lookup,
                uint32_t* brick_coord, uint32_t* brick_occ) {
    const size_t D = s->desc.size();
    for (size_t i = 0; i < D; ++i) {
        if (nodes) {
            nodes[2 * i] = s->desc[i].childPointer;
            nodes[2 * i + 1] = uint32_t(s->desc[i].validMask) | (uint32_t(s->desc[i].leafMask) << 8);
        }
        if (node_brick) node_brick[i] = s->desc[i].brickIndex;
    }
    const size_t bpa = size_t(s->bricksPerAxis);
    if (grid_lookup) {
        std::fill(grid_lookup, grid_lookup + bpa * bpa * bpa, NONE);
        // VoxelSceneCacher::BuildBrickGridLookup (VoxelSceneCacher.cpp:670-713)
        for (const auto& [key, idx] : s->brickGridToBrickView) {
            size_t bx = key & 0x3FF, by = (key >> 10) & 0x3FF, bz = (key >> 20) & 0x3FF;
            size_t li = bx + by * bpa + bz * bpa * bpa;
            if (li < bpa * bpa * bpa) grid_lookup[li] = idx;
        }
    }
    for (size_t b = 0; b < s->brickGrid.size(); ++b) {
        const I3 g = s->brickGrid[b];
        if (brick_coord) brick_coord[b] = uint32_t(g.x) | (uint32_t(g.y) << 10) | (uint32_t(g.z) << 20);
        if (brick_occ) {
            uint32_t* w = brick_occ + 16 * b;
            std::fill(w, w + 16, 0u);
            for (int z = 0; z < 8; ++z)
                for (int y = 0; y < 8; ++y)
                    for (int x = 0; x < 8; ++x)
                        if (s->brickVoxelOccupied(uint32_t(b), x, y, z, nullptr)) {
                            int i = z * 64 + y * 8 + x;
                            w[i >> 5] |= 1u << (i & 31);
                        }
        }
    }
}

namespace {
void cast_rays_impl(const vxo_scene* s, const float* rays, uint64_t n, float t_min, float t_max, vxo_hit* out,
                    int nthreads, const Lod* lod) {
    auto work = [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; ++i) {
            const float* r = rays + 6 * i;
            uint32_t iters = 0;
            Counters cnt;
            Hit h = castRay(*s, V3{r[0], r[1], r[2]}, V3{r[3], r[4], r[5]}, t_min, t_max, iters, cnt, lod);
            vxo_hit& o = out[i];
            o.t = h.hit ? h.tMin : 0.0f;
            o.t_exit = h.hit ? h.tMax : 0.0f;
            o.hit_point[0] = h.hitPoint.x; o.hit_point[1] = h.hitPoint.y; o.hit_point[2] = h.hitPoint.z;
            o.normal[0] = h.normal.x; o.normal[1] = h.normal.y; o.normal[2] = h.normal.z;
            o.brick = h.hit ? h.brick : NONE;
            o.node = h.hit ? h.node : NONE;
            o.voxel = h.hit ? h.voxel : 0xFFFFu;
            o.key[0] = h.key.x; o.key[1] = h.key.y; o.key[2] = h.key.z;
            o.scale = h.scale;
            o.flags = h.flags;
            o.iters = iters;
            o.grid_reads = cnt.grid_reads;
            o.dda_steps = cnt.dda_steps;
            o.leaf_visits = cnt.leaf_visits;
        }
    };
    int T = nthreads > 0 ? nthreads : int(std::max(1u, std::thread::hardware_concurrency()));
    if (T <= 1 || n < 1024) { work(0, n); return; }
    std::vector<std::thread> th;
    uint64_t chunk = (n + uint64_t(T) - 1) / uint64_t(T);
    for (int t = 0; t < T; ++t) {
        uint64_t b = uint64_t(t) * chunk, e = std::min(n, b + chunk);
        if (b >= e) break;
        th.emplace_back(work, b, e);
    }
    for (auto& x : th) x.join();
}
}  // namespace

void vxo_cast_rays(const vxo_scene* s, const float* rays, uint64_t n, float t_min, float t_max, vxo_hit* out,
                   int nthreads) {
    cast_rays_impl(s, rays, n, t_min, t_max, out, nthreads, nullptr);
}

void vxo_cast_rays_lod(const vxo_scene* s, const float* rays, uint64_t n, float t_min, float t_max,
                       float ray_orig_size, float ray_dir_size, vxo_hit* out, int nthreads) {
    Lod lod;
    lod.rayOrigSize = ray_orig_size;
    lod.rayDirSize = ray_dir_size;
    cast_rays_impl(s, rays, n, t_min, t_max, out, nthreads, &lod);
}

// Primary rays of the compute shader: the pixel uv of VoxelRayMarch.comp:453-455,
// uv = (vec2(pixel) + 0.5) / vec2(imageSize), and getRayDir
// (shaders/RayGeneration.glsl:61-71) with the push constants of
// VoxelRayMarch.comp:85-94 (pc: 16 words, fov in degrees).  Expressions are
// evaluated left to right as GLSL writes them; normalize is glm's
// v * (1 / sqrt(dot(v, v))) (the CPU column), radians(x) = x * (pi / 180).
// out: w * h rays {origin, direction}, row-major from the top row; uv_y
// (optional): each pixel's uv.y, which the miss colour reads.
void vxo_camera_rays(const float pc[16], uint32_t w, uint32_t h, float* out, float* uv_y) {
    const V3 camPos{pc[0], pc[1], pc[2]}, camDir{pc[4], pc[5], pc[6]};
    const V3 camUp{pc[8], pc[9], pc[10]}, camRight{pc[12], pc[13], pc[14]};
    const float fov = pc[7], aspect = pc[11];
    const float tanHalfFov = std::tan((fov * 0.5f) * 0.0174532925199432957692f);
    for (uint32_t py = 0; py < h; ++py)
        for (uint32_t px = 0; px < w; ++px) {
            const float uvx = (float(px) + 0.5f) / float(w);
            const float uvy = (float(py) + 0.5f) / float(h);
            const float ndcx = uvx * 2.0f - 1.0f;
            const float ndcy = -(uvy * 2.0f - 1.0f);
            const V3 rayDir = (camDir + ((camRight * ndcx) * tanHalfFov) * aspect) + (camUp * ndcy) * tanHalfFov;
            const float inv = 1.0f / std::sqrt(dot(rayDir, rayDir));
            const V3 d = rayDir * inv;
            float* r = out + (uint64_t(py) * w + px) * 6;
            r[0] = camPos.x; r[1] = camPos.y; r[2] = camPos.z;
            r[3] = d.x; r[4] = d.y; r[5] = d.z;
            if (uv_y) uv_y[uint64_t(py) * w + px] = uvy;
        }
}

// LODParameters::fromCameraWithNearPlane (SVOLOD.h:105-119); near_plane = 0
// gives fromCamera (:83-92).
void vxo_lod_from_camera(float fov_y, int32_t screen_height, float near_plane, float out[2]) {
    float pixelAngle = fov_y / static_cast<float>(screen_height);
    float dirSize = 2.0f * ::tanf(pixelAngle * 0.5f);
    out[0] = near_plane * dirSize;
    out[1] = dirSize;
}

// LODParameters::withBias (SVOLOD.h:169-176)
void vxo_lod_with_bias(const float in[2], float bias, float out[2]) {
    float multiplier = ::powf(2.0f, bias);
    out[0] = in[0] * multiplier;
    out[1] = in[1] * multiplier;
}

// DXT1ColorCompressor::decodeColorHead (DXT1Compressor.cpp:14-36)
void vxo_dxt1_decode_head(uint32_t head, float ref[12]) {
    const float scale = 1.0f / 4294967296.0f;
    V3 r0{float(head << 16) * scale, float(head << 21) * scale, float(head << 27) * scale};
    V3 r1{float(head) * scale, float(head << 5) * scale, float(head << 11) * scale};
    V3 r2 = r0 * (2.0f / 3.0f) + r1 * (1.0f / 3.0f);
    V3 r3 = r0 * (1.0f / 3.0f) + r1 * (2.0f / 3.0f);
    const V3 rr[4] = {r0, r1, r2, r3};
    for (int i = 0; i < 4; ++i) { ref[3 * i] = rr[i].x; ref[3 * i + 1] = rr[i].y; ref[3 * i + 2] = rr[i].z; }
}

// DXT1ColorCompressor::decodeBlockTyped (DXT1Compressor.cpp:113-130)
void vxo_dxt1_decode_block(uint64_t block, float out[48]) {
    uint32_t head = uint32_t(block);
    uint32_t bits = uint32_t(block >> 32);
    float ref[12];
    vxo_dxt1_decode_head(head, ref);
    for (int i = 0; i < 16; ++i) {
        const float* c = ref + 3 * (bits & 3);
        out[3 * i] = c[0]; out[3 * i + 1] = c[1]; out[3 * i + 2] = c[2];
        bits >>= 2;
    }
}

// DXT1ColorCompressor::encodeColorHead (DXT1Compressor.cpp:38-55)
uint32_t vxo_dxt1_encode_head(const float c0[3], const float c1[3]) {
    auto q = [](float v, float m, float sub, int hi) -> uint32_t {
        return uint32_t(std::clamp(f2i(v * m + 0.5f - sub), 0, hi));
    };
    uint32_t head = 0;
    head = uint32_t(std::clamp(f2i(c0[2] * 31.0f + 0.5f), 0, 31));
    head |= q(c0[1], 63.0f, float(head) * std::exp2(-5.0f), 63) << 5;
    head |= q(c0[0], 31.0f, float(head) * std::exp2(-11.0f), 31) << 11;
    head |= q(c1[2], 31.0f, float(head) * std::exp2(-16.0f), 31) << 16;
    head |= q(c1[1], 63.0f, float(head) * std::exp2(-21.0f), 63) << 21;
    head |= q(c1[0], 31.0f, float(head) * std::exp2(-27.0f), 31) << 27;
    return head;
}

// DXT1ColorCompressor::encodeBlockTyped (DXT1Compressor.cpp:57-111)
uint64_t vxo_dxt1_encode_block(const float* colors, uint64_t validCount, const int32_t* indices) {
    if (validCount == 0) return 0;
    auto C = [&](uint64_t i) { return V3{colors[3 * i], colors[3 * i + 1], colors[3 * i + 2]}; };
    int refIdx0 = 0, refIdx1 = 0;
    float maxDistSq = -std::numeric_limits<float>::max();
    for (uint64_t i = 0; i < validCount; ++i)
        for (uint64_t j = i + 1; j < validCount; ++j) {
            V3 diff = C(i) - C(j);
            float distSq = dot(diff, diff);
            if (distSq > maxDistSq) { refIdx0 = int(i); refIdx1 = int(j); maxDistSq = distSq; }
        }
    const float* c0 = colors + 3 * refIdx0;
    const float* c1 = colors + 3 * refIdx1;
    uint32_t head = vxo_dxt1_encode_head(c0, c1);
    float ref[12];
    vxo_dxt1_decode_head(head, ref);
    uint32_t bits = 0;
    for (uint64_t i = 0; i < validCount; ++i) {
        int bestIdx = 0;
        float bestDistSq = std::numeric_limits<float>::max();
        for (int j = 0; j < 4; ++j) {
            V3 diff = C(i) - V3{ref[3 * j], ref[3 * j + 1], ref[3 * j + 2]};
            float distSq = dot(diff, diff);
            if (distSq < bestDistSq) { bestIdx = j; bestDistSq = distSq; }
        }
        int texelIdx = indices ? indices[i] : int(i);
        bits |= uint32_t(bestIdx) << (texelIdx * 2);
    }
    return uint64_t(head) | (uint64_t(bits) << 32);
}

void vxo_hit_texel_dxt(const uint64_t* brick_dxt, uint32_t brick, uint32_t voxel, float out[3]) {
    uint64_t block = brick_dxt[uint64_t(brick) * 32 + (voxel >> 4)];
    float ref[12];
    vxo_dxt1_decode_head(uint32_t(block), ref);
    uint32_t sel = (uint32_t(block >> 32) >> ((voxel & 15) * 2)) & 3;
    out[0] = ref[3 * sel]; out[1] = ref[3 * sel + 1]; out[2] = ref[3 * sel + 2];
}

// vxo_hit_texel_dxt over n hit records; misses (brick 0xFFFFFFFF) give zeros.
void vxo_hit_texels_dxt(const uint64_t* brick_dxt, uint64_t n, const uint32_t* brick, const uint32_t* voxel,
                        float* out) {
    for (uint64_t i = 0; i < n; ++i) {
        if (brick[i] == 0xFFFFFFFFu) {
            out[3 * i] = out[3 * i + 1] = out[3 * i + 2] = 0.0f;
        } else {
            vxo_hit_texel_dxt(brick_dxt, brick[i], voxel[i], out + 3 * i);
        }
    }
}

// computeLighting (shaders/Lighting.glsl:19-28); sky colour (VoxelRayMarch.comp:493-499).
uint32_t vxo_shade(const float color[3], int hit, int normal_axis, int normal_neg, float uv_y) {
    V3 c;
    if (hit) {
        V3 L = normalize(V3{1.0f, 1.0f, -1.0f});
        V3 nrm{0, 0, 0};
        nrm[normal_axis] = normal_neg ? -1.0f : 1.0f;
        float diffuse = gmax(dot(nrm, L), 0.0f) * 0.7f;
        float k = 0.3f + diffuse;
        c = V3{color[0], color[1], color[2]} * k;
    } else {
        c = V3{0.5f, 0.7f, 1.0f} * (1.0f - uv_y * 0.5f);
    }
    auto u8 = [](float v) -> uint32_t {
        float cl = gmin(gmax(v, 0.0f), 1.0f);
        return uint32_t(cl * 255.0f + 0.5f);
    };
    return u8(c.x) | (u8(c.y) << 8) | (u8(c.z) << 16) | (255u << 24);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// DXT normal blocks: DXTNormalCompressor (VoxelData/src/Compression/
// DXT1Compressor.cpp:168-354), the geometric normals the rebuild encodes
// (SVO/src/SVORebuild.cpp:145-220, 615-722) and the decode of the compressed
// shader (shaders/Compression.glsl:115-177, VoxelRayMarch_Compressed.comp:160-165).
// Integer <-> float conversions are C++'s (round to nearest for int -> float,
// truncation for float -> int); int32 left shifts wrap.
// ---------------------------------------------------------------------------
namespace {

constexpr float NORMAL_COEFS[4] = {-1.0f, -1.0f / 3.0f, 1.0f / 3.0f, 1.0f};  // DXT1Compressor.h:130

inline int32_t shl32(int32_t v, int s) { return static_cast<int32_t>(static_cast<uint32_t>(v) << s); }
inline V3 neg(V3 v) { return {-v.x, -v.y, -v.z}; }
inline int iclamp1(int v, int lo, int hi) { return v < lo ? lo : (hi < v ? hi : v); }  // std::clamp

// DXTNormalCompressor::encodeRawNormal (DXT1Compressor.cpp:168-193)
uint32_t encodeRawNormal(V3 normal) {
    V3 a{std::abs(normal.x), std::abs(normal.y), std::abs(normal.z)};
    float myz = (a.y < a.z) ? a.z : a.y;  // std::max(a.y, a.z)
    int axis = (a.x >= myz) ? 0 : (a.y >= a.z) ? 1 : 2;
    V3 tuv = axis == 0 ? normal : axis == 1 ? V3{normal.y, normal.z, normal.x} : V3{normal.z, normal.x, normal.y};
    uint32_t result = 0;
    if (tuv.x < 0.0f) result |= 0x80000000u;
    result |= uint32_t(axis) << 29;
    float absT = std::abs(tuv.x);
    if (absT > 0.0f) {
        int u = iclamp1(f2i((tuv.y / absT) * 16383.0f), -0x4000, 0x3FFF);
        int v = iclamp1(f2i((tuv.z / absT) * 8191.0f), -0x2000, 0x1FFF);
        result |= uint32_t(u & 0x7FFF) << 14;
        result |= uint32_t(v & 0x3FFF);
    }
    return result;
}

// DXTNormalCompressor::decodeRawNormal (:195-207); Compression.glsl:115-138
V3 decodeRawNormal(uint32_t value) {
    int32_t sign = static_cast<int32_t>(value) >> 31;
    int axis = int((value >> 29) & 3u);
    int32_t t = sign ^ 0x7FFFFFFF;
    int32_t u = static_cast<int32_t>(value << 3);
    int32_t v = static_cast<int32_t>(value << 18);
    if (axis == 0) return V3{float(t), float(u), float(v)};
    if (axis == 1) return V3{float(v), float(t), float(u)};
    return V3{float(u), float(v), float(t)};
}

// DXTNormalCompressor::encodeNormalAxis (:209-228).  std::exp2 of the integer
// exponents here is an exact power of two (std::ldexp).
uint32_t encodeNormalAxis(uint32_t headUV, V3 axis, int shift) {
    float ax = std::abs(axis.x), ay = std::abs(axis.y), az = std::abs(axis.z);
    float maxComp = ax;  // std::max({...}): the first largest
    if (maxComp < ay) maxComp = ay;
    if (maxComp < az) maxComp = az;
    int exponent = 0;
    if (maxComp > 0.0f) {
        uint32_t bits;
        std::memcpy(&bits, &maxComp, sizeof(bits));
        exponent = iclamp1(static_cast<int>(bits >> 23) + (-127 - 31 + 1 - 3 + 13), 0, 15);
    }
    V3 scaled = axis * std::ldexp(1.0f, -exponent + (13 - 31));
    headUV |= uint32_t(exponent) << shift;
    headUV |= uint32_t(iclamp1(f2i((scaled.z + 8.5f) - float(headUV) * std::ldexp(1.0f, -4 - shift)), 0, 15) ^ 8)
              << (4 + shift);
    headUV |= uint32_t(iclamp1(f2i((scaled.y + 8.5f) - float(headUV) * std::ldexp(1.0f, -8 - shift)), 0, 15) ^ 8)
              << (8 + shift);
    headUV |= uint32_t(iclamp1(f2i((scaled.x + 8.5f) - float(headUV) * std::ldexp(1.0f, -12 - shift)), 0, 15) ^ 8)
              << (12 + shift);
    return headUV;
}

// DXTNormalCompressor::decodeNormalAxis (:230-240); Compression.glsl:140-156
V3 decodeNormalAxis(uint32_t headUV, int shift) {
    int32_t shifted = shl32(static_cast<int32_t>(headUV), 16 - shift);
    int exponent = (shifted >> 16) & 15;
    float scale = std::ldexp(1.0f, exponent + (3 - 13));
    return V3{float(shifted) * scale, float(shl32(shifted, 4)) * scale, float(shl32(shifted, 8)) * scale};
}

// DXTNormalCompressor::encodeBlockTyped (:242-333) over 16 normals.
void encodeNormalBlock(const V3* normals, size_t validCount, const int32_t* indices, uint64_t& blockA,
                       uint64_t& blockB) {
    blockA = blockB = 0;
    if (validCount == 0) return;
    V3 base = normals[0];
    for (size_t i = 1; i < validCount; ++i) base = base + normals[i];
    float baseLen = length(base);
    if (baseLen < 0.1f * static_cast<float>(validCount)) {
        int bestIdx = 0;
        float bestDot = dot(normals[0], base);
        for (size_t i = 1; i < validCount; ++i) {
            float d = dot(normals[i], base);
            if (d > bestDot) { bestIdx = int(i); bestDot = d; }
        }
        base = normals[bestIdx];
    }
    uint32_t headBase = encodeRawNormal(base);
    base = decodeRawNormal(headBase);
    int uIdx = 0;
    float uDot = dot(normals[0], base);
    for (size_t i = 1; i < validCount; ++i) {
        float d = dot(normals[i], base);
        if (d < uDot) { uIdx = int(i); uDot = d; }
    }
    uint32_t headUV = encodeNormalAxis(0, normals[uIdx] * length(base) - base, 0);
    V3 u = decodeNormalAxis(headUV, 0);
    V3 uRef[4];
    for (int i = 0; i < 4; ++i) uRef[i] = normalize(base + u * NORMAL_COEFS[i]);
    int vIdx = 0, vLerpIdx = 0;
    float vDot = std::numeric_limits<float>::max();
    for (size_t i = 0; i < validCount; ++i) {
        int bestLerp = 0;
        float bestDot = dot(normals[i], uRef[0]);
        for (int j = 1; j < 4; ++j) {
            float d = dot(normals[i], uRef[j]);
            if (d > bestDot) { bestLerp = j; bestDot = d; }
        }
        if (bestDot < vDot) { vIdx = int(i); vLerpIdx = bestLerp; vDot = bestDot; }
    }
    V3 tmp = base + u * NORMAL_COEFS[vLerpIdx];
    headUV = encodeNormalAxis(headUV, normals[vIdx] * length(tmp) - tmp, 16);
    V3 v = decodeNormalAxis(headUV, 16);
    V3 uvRef[16];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) uvRef[i + j * 4] = normalize((base + u * NORMAL_COEFS[i]) + v * NORMAL_COEFS[j]);
    uint32_t bitsU = 0, bitsV = 0;
    for (size_t i = 0; i < validCount; ++i) {
        int bestLerp = 0;
        float bestDot = dot(normals[i], uvRef[0]);
        for (int j = 1; j < 16; ++j) {
            float d = dot(normals[i], uvRef[j]);
            if (d > bestDot) { bestLerp = j; bestDot = d; }
        }
        int texelIdx = indices ? indices[i] : int(i);
        bitsU |= uint32_t(bestLerp & 3) << (texelIdx * 2);
        bitsV |= uint32_t(bestLerp >> 2) << (texelIdx * 2);
    }
    blockA = uint64_t(headBase) | (uint64_t(bitsU) << 32);
    blockB = uint64_t(headUV) | (uint64_t(bitsV) << 32);
}

// decodeBlockTyped (:335-354) / decodeDXTNormal (Compression.glsl:158-177) of one texel.
V3 decodeNormalTexel(uint64_t blockA, uint64_t blockB, int texel) {
    V3 base = decodeRawNormal(uint32_t(blockA));
    V3 u = decodeNormalAxis(uint32_t(blockB), 0);
    V3 v = decodeNormalAxis(uint32_t(blockB), 16);
    float cu = NORMAL_COEFS[(uint32_t(blockA >> 32) >> (texel * 2)) & 3u];
    float cv = NORMAL_COEFS[(uint32_t(blockB >> 32) >> (texel * 2)) & 3u];
    return (base + u * cu) + v * cv;
}

// getOccupancy / computeGeometricNormal (SVORebuild.cpp:145-193): central
// differences of the brick's occupancy, out-of-brick neighbours empty.
V3 geometricNormal(const uint32_t* occ, int x, int y, int z) {
    auto o = [&](int X, int Y, int Z) -> float {
        if (X < 0 || X >= 8 || Y < 0 || Y >= 8 || Z < 0 || Z >= 8) return 0.0f;
        int i = Z * 64 + Y * 8 + X;
        return ((occ[i >> 5] >> (i & 31)) & 1u) ? 1.0f : 0.0f;
    };
    V3 g{o(x + 1, y, z) - o(x - 1, y, z), o(x, y + 1, z) - o(x, y - 1, z), o(x, y, z + 1) - o(x, y, z - 1)};
    float len = length(g);
    if (len > 0.001f) return neg(normalize(g));
    return V3{0.0f, 1.0f, 0.0f};
}

// The normal half of the rebuild's per-brick compression (SVORebuild.cpp:658-722):
// empty texels carry (0,1,0); a block with an occupied texel is encoded over
// all 16 texels, an empty block is {0, 0}.
void brickNormalBlocks(const uint32_t* occ, uint64_t* out /* 64 u64 */) {
    V3 nrm[512];
    for (int i = 0; i < 512; ++i) nrm[i] = geometricNormal(occ, i & 7, (i >> 3) & 7, i >> 6);
    for (int b = 0; b < 32; ++b) {
        V3 bn[16];
        int valid = 0;
        for (int t = 0; t < 16; ++t) {
            int i = b * 16 + t;
            bool occd = (occ[i >> 5] >> (i & 31)) & 1u;
            bn[t] = occd ? nrm[i] : V3{0.0f, 1.0f, 0.0f};
            valid += occd;
        }
        if (valid) encodeNormalBlock(bn, 16, nullptr, out[2 * b], out[2 * b + 1]);
        else out[2 * b] = out[2 * b + 1] = 0;
    }
}

}  // namespace

extern "C" {

void vxo_dxtn_encode_block(const float* normals, uint64_t valid_count, const int32_t* indices, uint64_t out[2]) {
    V3 n[16];
    for (uint64_t i = 0; i < valid_count && i < 16; ++i) n[i] = V3{normals[3 * i], normals[3 * i + 1], normals[3 * i + 2]};
    encodeNormalBlock(n, size_t(valid_count < 16 ? valid_count : 16), indices, out[0], out[1]);
}

void vxo_dxtn_decode_block(const uint64_t in[2], float out[48]) {
    for (int t = 0; t < 16; ++t) {
        V3 v = decodeNormalTexel(in[0], in[1], t);
        out[3 * t] = v.x; out[3 * t + 1] = v.y; out[3 * t + 2] = v.z;
    }
}

uint32_t vxo_encode_raw_normal(const float n[3]) { return encodeRawNormal(V3{n[0], n[1], n[2]}); }

void vxo_geometric_normals(const uint32_t* occ, float out[1536]) {
    for (int i = 0; i < 512; ++i) {
        V3 v = geometricNormal(occ, i & 7, (i >> 3) & 7, i >> 6);
        out[3 * i] = v.x; out[3 * i + 1] = v.y; out[3 * i + 2] = v.z;
    }
}

void vxo_brick_normals(const uint32_t* occ, uint64_t brick_count, uint64_t* out, int nthreads) {
    auto work = [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; ++i) brickNormalBlocks(occ + 16 * i, out + 64 * i);
    };
    int T = nthreads > 0 ? nthreads : int(std::max(1u, std::thread::hardware_concurrency()));
    if (T <= 1 || brick_count < 64) { work(0, brick_count); return; }
    std::vector<std::thread> th;
    uint64_t chunk = (brick_count + uint64_t(T) - 1) / uint64_t(T);
    for (int t = 0; t < T; ++t) {
        uint64_t b = uint64_t(t) * chunk, e = std::min(brick_count, b + chunk);
        if (b >= e) break;
        th.emplace_back(work, b, e);
    }
    for (auto& x : th) x.join();
}

// getCompressedVoxelNormal (VoxelRayMarch_Compressed.comp:160-165): the
// normalised decode of the hit voxel's texel.
void vxo_hit_normal_dxt(const uint64_t* brick_nrm, uint32_t brick, uint32_t voxel, float out[3]) {
    const uint64_t* blk = brick_nrm + (uint64_t(brick) * 32 + (voxel >> 4)) * 2;
    V3 v = normalize(decodeNormalTexel(blk[0], blk[1], int(voxel & 15)));
    out[0] = v.x; out[1] = v.y; out[2] = v.z;
}

// Compressed shading of a hit: n = normalize(n_dxt + n_face * 0.5) (the blend of
// VoxelRayMarch_Compressed.comp:242-256 with the hit's entry-face normal as the
// DDA normal), then computeLighting (Lighting.glsl:19-28).  Miss: sky.
uint32_t vxo_shade_dxt_normal(const float color[3], int hit, const float n_dxt[3], int normal_axis, int normal_neg,
                              float uv_y) {
    V3 c;
    if (hit) {
        V3 face{0, 0, 0};
        face[normal_axis] = normal_neg ? -1.0f : 1.0f;
        V3 n = normalize(V3{n_dxt[0], n_dxt[1], n_dxt[2]} + face * 0.5f);
        V3 L = normalize(V3{1.0f, 1.0f, -1.0f});
        float k = 0.3f + gmax(dot(n, L), 0.0f) * 0.7f;
        c = V3{color[0], color[1], color[2]} * k;
    } else {
        c = V3{0.5f, 0.7f, 1.0f} * (1.0f - uv_y * 0.5f);
    }
    auto u8 = [](float v) -> uint32_t {
        float cl = gmin(gmax(v, 0.0f), 1.0f);
        return uint32_t(cl * 255.0f + 0.5f);
    };
    return u8(c.x) | (u8(c.y) << 8) | (u8(c.z) << 16) | (255u << 24);
}

}  // extern "C"

// The colour half of the rebuild's per-brick compression (SVORebuild.cpp:658-722):
// empty texels are (0,0,0); a block with an occupied texel is encoded over all
// 16 texels (encodeBlockTyped(blockColors, 16, nullptr)), an empty block is 0.
extern "C" void vxo_brick_dxt1(const float* rgb, const uint32_t* occ, uint64_t brick_count, uint64_t* out) {
    for (uint64_t b = 0; b < brick_count; ++b)
        for (int k = 0; k < 32; ++k) {
            float cols[48];
            bool any = false;
            for (int t = 0; t < 16; ++t) {
                const int i = k * 16 + t;
                const bool o = (occ[b * 16 + (i >> 5)] >> (i & 31)) & 1u;
                any = any || o;
                for (int c = 0; c < 3; ++c) cols[3 * t + c] = o ? rgb[(b * 512 + i) * 3 + c] : 0.0f;
            }
            out[b * 32 + k] = any ? vxo_dxt1_encode_block(cols, 16, nullptr) : 0;
        }
}
