// vx_cache.cpp - scene cache files: this library's exact format (VXSC) and the
// reference's VoxelSceneCacher format (VSCA version 1,
// CashSystem/src/VoxelSceneCacher.cpp:179-364), both as host arrays that
// vx_scene_create uploads, so a benchmark can skip the octree build.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "vx_internal.h"

struct vx_cache {
    vx_octree_config cfg{};
    std::vector<uint32_t> nodes, node_brick, grid, coord, occ;
    int32_t color_kind = VX_COLOR_NONE;
    std::vector<uint8_t> color, normal;
    std::vector<uint32_t> materials;  // a VSCA file's brickData words (512 per brick), or empty
};

namespace {

using vx::fail;

constexpr uint32_t VXSC_MAGIC = 0x43535856u;  // "VXSC"
constexpr uint32_t VXSC_VERSION = 1;
constexpr uint32_t VSCA_MAGIC = 0x56534341u;  // VOXEL_SCENE_CACHE_MAGIC (VoxelSceneCacher.cpp:181)
constexpr uint32_t VSCA_VERSION = 1;          // VOXEL_SCENE_CACHE_VERSION (:180)

// 64-bit FNV-1a over the 32-bit words of the payload sections of a VXSC file
// (every section is a whole number of words).
struct Fnv {
    uint64_t h = 0xCBF29CE484222325ULL;
    void add(const void* p, size_t n) {
        const uint8_t* b = static_cast<const uint8_t*>(p);
        for (size_t i = 0; i + 4 <= n; i += 4) {
            uint32_t w;
            std::memcpy(&w, b + i, 4);
            h = (h ^ w) * 0x100000001B3ULL;
        }
    }
};

struct File {
    FILE* f = nullptr;
    ~File() {
        if (f) std::fclose(f);
    }
};

// Bytes left to read in f (sizes in a file are checked against this before
// anything is allocated for them).
uint64_t remaining(FILE* f) {
    const long here = std::ftell(f);
    if (here < 0 || std::fseek(f, 0, SEEK_END) != 0) return 0;
    const long end = std::ftell(f);
    std::fseek(f, here, SEEK_SET);
    return end > here ? uint64_t(end - here) : 0;
}

bool put(FILE* f, const void* p, size_t n) { return n == 0 || std::fwrite(p, 1, n, f) == n; }
bool get(FILE* f, void* p, size_t n) { return n == 0 || std::fread(p, 1, n, f) == n; }
template <class T>
bool put_v(FILE* f, const T& v) { return put(f, &v, sizeof(T)); }
template <class T>
bool get_v(FILE* f, T& v) { return get(f, &v, sizeof(T)); }

uint64_t color_bytes_per_brick(int32_t kind) {
    return (kind == VX_COLOR_RGBA8 || kind == VX_COLOR_MATERIAL) ? 512 * 4 : kind == VX_COLOR_DXT1 ? 32 * 8 : 0;
}

// Host copies of a vx_scene_desc's arrays, after the checks vx_scene_create
// would make on sizes.
int cache_from_desc(const vx_scene_desc* d, vx_cache& c, const char* what) {
    if (!d) return fail(VX_EINVAL, std::string(what) + ": null desc");
    const uint64_t bpa = uint64_t(d->config.bricks_per_axis);
    if (d->config.bricks_per_axis < 1 || d->config.bricks_per_axis > 1024)
        return fail(VX_EINVAL, std::string(what) + ": bricks_per_axis out of range");
    if ((d->node_count && (!d->nodes || !d->node_brick)) || !d->grid_lookup ||
        (d->brick_count && (!d->brick_coord || !d->brick_occ)))
        return fail(VX_EINVAL, std::string(what) + ": missing arrays");
    c.cfg = d->config;
    const uint32_t* nodes = reinterpret_cast<const uint32_t*>(d->nodes);
    c.nodes.assign(nodes, nodes + 2 * uint64_t(d->node_count));
    c.node_brick.assign(d->node_brick, d->node_brick + d->node_count);
    c.grid.assign(d->grid_lookup, d->grid_lookup + bpa * bpa * bpa);
    c.coord.assign(d->brick_coord, d->brick_coord + d->brick_count);
    c.occ.assign(d->brick_occ, d->brick_occ + 16 * uint64_t(d->brick_count));
    c.color_kind = d->brick_color ? d->color_kind : VX_COLOR_NONE;
    const uint64_t cb = color_bytes_per_brick(c.color_kind) * d->brick_count;
    if (cb) {
        const uint8_t* p = static_cast<const uint8_t*>(d->brick_color);
        c.color.assign(p, p + cb);
    }
    if (d->brick_normal) {
        const uint8_t* p = static_cast<const uint8_t*>(d->brick_normal);
        c.normal.assign(p, p + 512 * uint64_t(d->brick_count));
    }
    return VX_OK;
}

// VoxelSceneCreateInfo::ComputeHash (VoxelSceneCacher.h:156-165)
uint64_t vsca_key(uint32_t scene_type, uint32_t resolution, float density, uint32_t seed) {
    const uint32_t dq = static_cast<uint32_t>(density * 100.0f);
    uint64_t h = scene_type;
    h = h * 31 + resolution;
    h = h * 31 + dq;
    h = h * 31 + seed;
    return h;
}

// OctreeConfig (VoxelSceneCacher.h:100-132): 256-byte UBO part + worldGridSize.
struct RefOctreeConfig {
    int32_t esvoMaxScale, userMaxLevels, brickDepthLevels, brickSize;
    int32_t minESVOScale, brickESVOScale, bricksPerAxis, padding1;
    float gridMin[3], padding2;
    float gridMax[3], padding3;
    float localToWorld[16], worldToLocal[16];
    float padding4[16];
    float worldGridSize;
};
static_assert(sizeof(RefOctreeConfig) == 260, "OctreeConfig is 260 bytes");

}  // namespace

extern "C" {

static int vx_cache_write_body(const char* path, const vx_scene_desc* d) {
    if (!path) return fail(VX_EINVAL, "vx_cache_write: null path");
    vx_cache c;
    if (int r = cache_from_desc(d, c, "vx_cache_write")) return r;
    File f;
    f.f = std::fopen(path, "wb");
    if (!f.f) return fail(VX_EIO, std::string("vx_cache_write: cannot open ") + path);
    const uint32_t D = uint32_t(c.node_brick.size()), B = uint32_t(c.coord.size());
    const uint32_t has_n = c.normal.empty() ? 0u : 1u;
    bool ok = put_v(f.f, VXSC_MAGIC) && put_v(f.f, VXSC_VERSION) && put_v(f.f, c.cfg) && put_v(f.f, D) && put_v(f.f, B) &&
              put_v(f.f, c.color_kind) && put_v(f.f, has_n);
    Fnv h;
    struct Sec { const void* p; uint64_t n; };
    const Sec secs[] = {{c.nodes.data(), c.nodes.size() * 4}, {c.node_brick.data(), c.node_brick.size() * 4},
                        {c.grid.data(), c.grid.size() * 4},   {c.coord.data(), c.coord.size() * 4},
                        {c.occ.data(), c.occ.size() * 4},     {c.color.data(), c.color.size()},
                        {c.normal.data(), c.normal.size()}};
    for (const Sec& s : secs) {
        ok = ok && put_v(f.f, s.n) && put(f.f, s.p, s.n);
        h.add(s.p, s.n);
    }
    ok = ok && put_v(f.f, h.h);
    if (!ok) return fail(VX_EIO, std::string("vx_cache_write: write failed: ") + path);
    return VX_OK;
}

int vx_cache_write(const char* path, const vx_scene_desc* d) {
    return vx::guarded("vx_cache_write", [&] { return vx_cache_write_body(path, d); });
}

static int vx_cache_read_body(const char* path, vx_cache** out) {
    if (!path || !out) return fail(VX_EINVAL, "vx_cache_read: null argument");
    *out = nullptr;
    File f;
    f.f = std::fopen(path, "rb");
    if (!f.f) return fail(VX_EIO, std::string("vx_cache_read: cannot open ") + path);
    auto c = std::make_unique<vx_cache>();
    uint32_t magic = 0, version = 0, D = 0, B = 0, has_n = 0;
    if (!get_v(f.f, magic) || magic != VXSC_MAGIC) return fail(VX_EFORMAT, "vx_cache_read: not a VXSC file");
    if (!get_v(f.f, version) || version != VXSC_VERSION) return fail(VX_EFORMAT, "vx_cache_read: unknown version");
    if (!get_v(f.f, c->cfg) || !get_v(f.f, D) || !get_v(f.f, B) || !get_v(f.f, c->color_kind) || !get_v(f.f, has_n))
        return fail(VX_EFORMAT, "vx_cache_read: truncated header");
    const int64_t bpa = c->cfg.bricks_per_axis;
    if (bpa < 1 || bpa > 1024 || has_n > 1 ||
        (color_bytes_per_brick(c->color_kind) == 0 && c->color_kind != VX_COLOR_NONE))
        return fail(VX_EFORMAT, "vx_cache_read: bad header");
    const uint64_t want[7] = {uint64_t(D) * 8, uint64_t(D) * 4, uint64_t(bpa * bpa * bpa) * 4, uint64_t(B) * 4,
                              uint64_t(B) * 64, color_bytes_per_brick(c->color_kind) * B, has_n ? uint64_t(B) * 512 : 0};
    uint64_t total = 0;
    for (uint64_t w : want) total += w + 8;
    if (total + 8 > remaining(f.f)) return fail(VX_EFORMAT, "vx_cache_read: the file is shorter than its header says");
    c->nodes.resize(2 * uint64_t(D));
    c->node_brick.resize(D);
    c->grid.resize(uint64_t(bpa * bpa * bpa));
    c->coord.resize(B);
    c->occ.resize(16 * uint64_t(B));
    c->color.resize(want[5]);
    c->normal.resize(want[6]);
    void* dst[7] = {c->nodes.data(), c->node_brick.data(), c->grid.data(), c->coord.data(),
                    c->occ.data(), c->color.data(), c->normal.data()};
    Fnv h;
    for (int i = 0; i < 7; ++i) {
        uint64_t n = 0;
        if (!get_v(f.f, n) || n != want[i]) return fail(VX_EFORMAT, "vx_cache_read: section size mismatch");
        if (!get(f.f, dst[i], n)) return fail(VX_EFORMAT, "vx_cache_read: truncated section");
        h.add(dst[i], n);
    }
    uint64_t sum = 0;
    if (!get_v(f.f, sum) || sum != h.h) return fail(VX_EFORMAT, "vx_cache_read: checksum mismatch");
    *out = c.release();
    return VX_OK;
}

int vx_cache_read(const char* path, vx_cache** out) {
    return vx::guarded("vx_cache_read", [&] { return vx_cache_read_body(path, out); });
}

// VoxelSceneCacher::SerializeToFile (VoxelSceneCacher.cpp:209-265) for one
// entry.  The reference's ChildDescriptor holds a 15-bit child pointer and no
// far pointers, so scenes whose child pointers reach 2^15 cannot be written
// (VX_EOVERFLOW) rather than truncated.  brickData holds the material words of
// a VX_COLOR_MATERIAL scene, else material 1 for every occupied voxel; the
// material table is written empty.
static int vx_cache_write_vsca_body(const char* path, const vx_scene_desc* d, uint32_t scene_type, uint32_t resolution,
                        float density, uint32_t seed) {
    if (!path) return fail(VX_EINVAL, "vx_cache_write_vsca: null path");
    vx_cache c;
    if (int r = cache_from_desc(d, c, "vx_cache_write_vsca")) return r;
    if (c.color_kind == VX_COLOR_RGBA8)
        return fail(VX_EINVAL, "vx_cache_write_vsca: the format holds DXT1 colours only");
    const uint64_t D = c.node_brick.size(), B = c.coord.size();
    std::vector<uint64_t> esvo(D);
    for (uint64_t i = 0; i < D; ++i) {
        const uint32_t cp = c.nodes[2 * i], masks = c.nodes[2 * i + 1];
        if (cp > 0x7FFFu) return fail(VX_EOVERFLOW, "vx_cache_write_vsca: child pointer exceeds 15 bits");
        if (c.node_brick[i] > 0xFFFFFFu) return fail(VX_EOVERFLOW, "vx_cache_write_vsca: brick index exceeds 24 bits");
        // ChildDescriptor (SVOTypes.h:36-47): childPointer:15 far:1 valid:8 leaf:8 | brickIndex:24 flags:8
        const uint32_t lo = cp | ((masks & 0xFFu) << 16) | (((masks >> 8) & 0xFFu) << 24);
        esvo[i] = uint64_t(lo) | (uint64_t(c.node_brick[i] & 0xFFFFFFu) << 32);
    }
    std::vector<uint32_t> brick_data(B * 512, 0u);
    uint32_t solid = 0;
    const uint32_t* words = c.color_kind == VX_COLOR_MATERIAL ? reinterpret_cast<const uint32_t*>(c.color.data())
                                                              : nullptr;
    for (uint64_t b = 0; b < B; ++b)
        for (uint32_t v = 0; v < 512; ++v)
            if ((c.occ[b * 16 + (v >> 5)] >> (v & 31)) & 1u) {
                brick_data[b * 512 + v] = words ? words[b * 512 + v] : 1u;
                if (brick_data[b * 512 + v] == 0u)
                    return fail(VX_EINVAL, "vx_cache_write_vsca: an occupied voxel has material word 0");
                ++solid;
            }
    if (words) c.color.clear();  // the words went into brickData; the file's colour section stays empty
    RefOctreeConfig oc;
    std::memset(&oc, 0, sizeof(oc));
    const int32_t L = c.cfg.max_levels;
    oc.esvoMaxScale = 22;
    oc.userMaxLevels = L;
    oc.brickDepthLevels = c.cfg.brick_depth;
    oc.brickSize = 1 << c.cfg.brick_depth;
    oc.minESVOScale = 22 - L + 1;
    oc.brickESVOScale = 22 - (L - 1 - (L - c.cfg.brick_depth));  // VoxelSceneCacher.cpp:597-599
    oc.bricksPerAxis = c.cfg.bricks_per_axis;
    for (int i = 0; i < 3; ++i) {
        oc.gridMin[i] = c.cfg.world_min[i];
        oc.gridMax[i] = c.cfg.world_max[i];
    }
    // localToWorld = translate(0) * scale(10) and its inverse (:611-622)
    for (int i = 0; i < 16; ++i) oc.localToWorld[i] = oc.worldToLocal[i] = 0.0f;
    for (int i = 0; i < 3; ++i) {
        oc.localToWorld[i * 5] = 10.0f;
        oc.worldToLocal[i * 5] = 1.0f / 10.0f;
    }
    oc.localToWorld[15] = oc.worldToLocal[15] = 1.0f;
    oc.worldGridSize = 10.0f;
    File f;
    f.f = std::fopen(path, "wb");
    if (!f.f) return fail(VX_EIO, std::string("vx_cache_write_vsca: cannot open ") + path);
    const uint32_t entries = 1;
    const uint64_t key = vsca_key(scene_type, resolution, density, seed);
    auto vec = [&](const void* p, uint64_t count, uint64_t elem) {
        return put_v(f.f, count) && put(f.f, p, count * elem);
    };
    const uint32_t nc = uint32_t(D), bc = uint32_t(B);
    bool ok = put_v(f.f, VSCA_MAGIC) && put_v(f.f, VSCA_VERSION) && put_v(f.f, entries) && put_v(f.f, key) &&
              put_v(f.f, scene_type) && put_v(f.f, resolution) && put_v(f.f, density) && put_v(f.f, seed) &&
              vec(esvo.data(), D * 8, 1) && vec(brick_data.data(), B * 2048, 1) && vec(nullptr, 0, 32) &&
              vec(c.color.data(), c.color.size(), 1) && vec(c.normal.data(), c.normal.size(), 1) &&
              vec(c.grid.data(), c.grid.size(), 4) && put_v(f.f, oc) && put_v(f.f, nc) && put_v(f.f, bc) &&
              put_v(f.f, solid) && put_v(f.f, resolution) && put_v(f.f, scene_type);
    if (!ok) return fail(VX_EIO, std::string("vx_cache_write_vsca: write failed: ") + path);
    return VX_OK;
}

int vx_cache_write_vsca(const char* path, const vx_scene_desc* d, uint32_t scene_type, uint32_t resolution,
                        float density, uint32_t seed) {
    return vx::guarded("vx_cache_write_vsca", [&] { return vx_cache_write_vsca_body(path, d, scene_type, resolution, density, seed); });
}

// VoxelSceneCacher::DeserializeFromFile (:267-364), entry `entry` of the
// file, into this library's arrays: descriptors as vx_nodes_from_reference
// converts them, occupancy = brickData word != 0 (the compressed shader's test,
// VoxelRayMarch_Compressed.comp), brick coordinates from brickGridLookup.
static int vx_cache_read_vsca_body(const char* path, uint32_t entry, vx_cache** out) {
    if (!path || !out) return fail(VX_EINVAL, "vx_cache_read_vsca: null argument");
    *out = nullptr;
    File f;
    f.f = std::fopen(path, "rb");
    if (!f.f) return fail(VX_EIO, std::string("vx_cache_read_vsca: cannot open ") + path);
    uint32_t magic = 0, version = 0, entries = 0;
    if (!get_v(f.f, magic) || magic != VSCA_MAGIC) return fail(VX_EFORMAT, "vx_cache_read_vsca: not a VSCA file");
    if (!get_v(f.f, version) || version != VSCA_VERSION) return fail(VX_EFORMAT, "vx_cache_read_vsca: unknown version");
    if (!get_v(f.f, entries) || entry >= entries) return fail(VX_EINVAL, "vx_cache_read_vsca: no such entry");
    auto rvec = [&](std::vector<uint8_t>& v, uint64_t elem) {
        uint64_t n = 0;
        if (!get_v(f.f, n) || n > (uint64_t(1) << 40) / elem || n * elem > remaining(f.f)) return false;
        v.resize(n * elem);
        return get(f.f, v.data(), v.size());
    };
    for (uint32_t e = 0; e <= entry; ++e) {
        uint64_t key = 0;
        uint32_t scene_type = 0, resolution = 0, seed = 0;
        float density = 0;
        std::vector<uint8_t> esvo, bricks, materials, colors, normals, grid;
        RefOctreeConfig oc;
        uint32_t nc = 0, bc = 0, solid = 0, res2 = 0, st2 = 0;
        bool ok = get_v(f.f, key) && get_v(f.f, scene_type) && get_v(f.f, resolution) && get_v(f.f, density) &&
                  get_v(f.f, seed) && rvec(esvo, 1) && rvec(bricks, 1) && rvec(materials, 32) && rvec(colors, 1) &&
                  rvec(normals, 1) && rvec(grid, 4) && get_v(f.f, oc) && get_v(f.f, nc) && get_v(f.f, bc) &&
                  get_v(f.f, solid) && get_v(f.f, res2) && get_v(f.f, st2);
        if (!ok) return fail(VX_EFORMAT, "vx_cache_read_vsca: truncated entry");
        if (key != vsca_key(scene_type, resolution, density, seed))
            return fail(VX_EFORMAT, "vx_cache_read_vsca: key mismatch");  // (:315-319)
        if (e != entry) continue;
        const int64_t bpa = oc.bricksPerAxis;
        if (bpa < 1 || bpa > 1024 || esvo.size() != uint64_t(nc) * 8 || bricks.size() != uint64_t(bc) * 2048 ||
            grid.size() != uint64_t(bpa * bpa * bpa) * 4 || (!colors.empty() && colors.size() != uint64_t(bc) * 256) ||
            (!normals.empty() && normals.size() != uint64_t(bc) * 512) || oc.brickDepthLevels != 3)
            return fail(VX_EFORMAT, "vx_cache_read_vsca: inconsistent sizes");
        auto c = std::make_unique<vx_cache>();
        for (int i = 0; i < 3; ++i) {
            c->cfg.world_min[i] = oc.gridMin[i];
            c->cfg.world_max[i] = oc.gridMax[i];
        }
        c->cfg.max_levels = oc.userMaxLevels;
        c->cfg.brick_depth = oc.brickDepthLevels;
        c->cfg.bricks_per_axis = oc.bricksPerAxis;
        c->nodes.resize(2 * uint64_t(nc));
        c->node_brick.resize(nc);
        if (nc && vx_nodes_from_reference(reinterpret_cast<const uint64_t*>(esvo.data()), nc,
                                          reinterpret_cast<vx_node*>(c->nodes.data()), c->node_brick.data()))
            return VX_EINVAL;
        c->grid.resize(grid.size() / 4);
        std::memcpy(c->grid.data(), grid.data(), grid.size());
        c->coord.assign(bc, 0xFFFFFFFFu);
        for (uint64_t s = 0; s < c->grid.size(); ++s) {
            const uint32_t b = c->grid[s];
            if (b == 0xFFFFFFFFu) continue;
            if (b >= bc || c->coord[b] != 0xFFFFFFFFu)
                return fail(VX_EFORMAT, "vx_cache_read_vsca: brickGridLookup is not a brick permutation");
            c->coord[b] = uint32_t(s % bpa) | (uint32_t((s / bpa) % bpa) << 10) | (uint32_t(s / (bpa * bpa)) << 20);
        }
        for (uint32_t b = 0; b < bc; ++b)
            if (c->coord[b] == 0xFFFFFFFFu) return fail(VX_EFORMAT, "vx_cache_read_vsca: brick missing from the grid");
        c->occ.assign(uint64_t(bc) * 16, 0u);
        const uint32_t* bd = reinterpret_cast<const uint32_t*>(bricks.data());
        for (uint64_t b = 0; b < bc; ++b)
            for (uint32_t v = 0; v < 512; ++v)
                if (bd[b * 512 + v]) c->occ[b * 16 + (v >> 5)] |= 1u << (v & 31);
        c->materials.assign(bd, bd + uint64_t(bc) * 512);
        if (!colors.empty()) {
            c->color_kind = VX_COLOR_DXT1;
            c->color = std::move(colors);
        }
        c->normal = std::move(normals);
        *out = c.release();
        return VX_OK;
    }
    return fail(VX_EINVAL, "vx_cache_read_vsca: no such entry");
}

int vx_cache_read_vsca(const char* path, uint32_t entry, vx_cache** out) {
    return vx::guarded("vx_cache_read_vsca", [&] { return vx_cache_read_vsca_body(path, entry, out); });
}

int vx_cache_desc(const vx_cache* c, vx_scene_desc* d) {
    if (!c || !d) return fail(VX_EINVAL, "vx_cache_desc: null argument");
    std::memset(d, 0, sizeof(*d));
    d->config = c->cfg;
    d->nodes = reinterpret_cast<const vx_node*>(c->nodes.data());
    d->node_count = uint32_t(c->node_brick.size());
    d->brick_count = uint32_t(c->coord.size());
    d->node_brick = c->node_brick.data();
    d->grid_lookup = c->grid.data();
    d->brick_coord = c->coord.data();
    d->brick_occ = c->occ.data();
    d->color_kind = c->color.empty() ? VX_COLOR_NONE : c->color_kind;
    d->brick_color = c->color.empty() ? nullptr : c->color.data();
    if (c->color.empty() && !c->materials.empty()) {
        d->color_kind = VX_COLOR_MATERIAL;
        d->brick_color = c->materials.data();
    }
    d->brick_normal = c->normal.empty() ? nullptr : c->normal.data();
    return VX_OK;
}

int vx_cache_desc_materials(const vx_cache* c, vx_scene_desc* d) {
    if (int r = vx_cache_desc(c, d)) return r;
    if (!c->materials.empty()) {
        d->color_kind = VX_COLOR_MATERIAL;
        d->brick_color = c->materials.data();
    } else if (c->color_kind != VX_COLOR_MATERIAL || c->color.empty()) {
        return fail(VX_EINVAL, "vx_cache_desc_materials: the cache holds no material words");
    }
    return VX_OK;
}

int vx_cache_free(vx_cache* c) {
    delete c;
    return VX_OK;
}

static int vx_scene_save_body(const vx_scene* s, const char* path) {
    vx_scene_info i{};
    if (int r = vx_scene_info_get(s, &i)) return r;
    vx_cache c;
    const uint64_t bpa = uint64_t(i.config.bricks_per_axis);
    c.cfg = i.config;
    c.nodes.resize(2 * uint64_t(i.node_count));
    c.node_brick.resize(i.node_count);
    c.grid.resize(bpa * bpa * bpa);
    c.coord.resize(i.brick_count);
    c.occ.resize(16 * uint64_t(i.brick_count));
    c.color_kind = i.color_kind;
    c.color.resize(color_bytes_per_brick(i.color_kind) * i.brick_count);
    c.normal.resize(i.has_normals ? 512 * uint64_t(i.brick_count) : 0);
    if (int r = vx_scene_download(s, c.nodes.data(), c.node_brick.data(), c.grid.data(), c.coord.data(), c.occ.data(),
                                  c.color.empty() ? nullptr : c.color.data(),
                                  c.normal.empty() ? nullptr : reinterpret_cast<uint64_t*>(c.normal.data())))
        return r;
    vx_scene_desc d;
    vx_cache_desc(&c, &d);
    return vx_cache_write(path, &d);
}

int vx_scene_save(const vx_scene* s, const char* path) {
    return vx::guarded("vx_scene_save", [&] { return vx_scene_save_body(s, path); });
}

static int vx_scene_load_body(const char* path, vx_scene** out) {
    if (!out) return fail(VX_EINVAL, "vx_scene_load: null argument");
    vx_cache* c = nullptr;
    if (int r = vx_cache_read(path, &c)) return r;
    vx_scene_desc d;
    vx_cache_desc(c, &d);
    const int r = vx_scene_create(&d, out);
    vx_cache_free(c);
    return r;
}

int vx_scene_load(const char* path, vx_scene** out) {
    return vx::guarded("vx_scene_load", [&] { return vx_scene_load_body(path, out); });
}

}  // extern "C"
