// vx_build.cpp - host scene builder, reference-descriptor conversion and
// seeded synthetic inputs.
//
// The builder produces the device layout of vx.h from a dense occupancy grid
// with world bounds [0,R]^3, matching LaineKarrasOctree::rebuild
// (SVO/src/SVORebuild.cpp:228-607) and VoxelSceneCacher::BuildOctree /
// BuildBrickGridLookup (CashSystem/src/VoxelSceneCacher.cpp:463-713) index for
// index.  Instead of the reference's hash maps and BFS queue it uses the
// equivalent closed form:
//  - brick index = rank of the brick's grid coordinate in Morton order
//    (SVORebuild.cpp:346-371; the 2^20 coordinate offset of MortonCode64 sets
//    the same top bit on every axis and does not change the order);
//  - the BFS of :540-598 visits the tree level by level, and inside a level in
//    the order (parent position, octant), which is the Morton order of the
//    node coordinates at that level; every parent's children are either all
//    bricks or all internal nodes, so "non-leaf children first" keeps octant
//    order.  Descriptor index = level offset + Morton rank in the level, and a
//    node's child pointer = offset of the level below + number of children of
//    the nodes before it.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "vx_hash.h"
#include "vx_internal.h"

namespace {

constexpr uint32_t NONE = 0xFFFFFFFFu;

using vx::morton3;

int hw_threads() {
    unsigned t = std::thread::hardware_concurrency();
    return t ? int(t) : 1;
}

template <class F>
void parallel_for(int64_t n, F&& f) {
    int T = int(std::min<int64_t>(hw_threads(), std::max<int64_t>(n, 1)));
    if (T <= 1) { for (int64_t i = 0; i < n; ++i) f(i); return; }
    std::atomic<int64_t> next{0};
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t)
        th.emplace_back([&] {
            for (int64_t i; (i = next.fetch_add(1)) < n;) f(i);
        });
    for (auto& x : th) x.join();
}

using vx::hash4;

}  // namespace

struct vx_build {
    uint32_t R = 0;
    vx_octree_config cfg{};
    std::vector<vx_node> nodes;
    std::vector<uint32_t> node_brick, grid, coord, occ;
};

extern "C" {

static int vx_build_dense_body(const uint64_t* bits, uint32_t R, int32_t max_levels, vx_build** out) {
    using namespace vx;
    if (!bits || !out) return fail(VX_EINVAL, "vx_build_dense: null argument");
    *out = nullptr;
    if (R < 64 || R % 64 != 0 || R > 8192)
        return fail(VX_EINVAL, "vx_build_dense: R must be a multiple of 64 in [64, 8192]");
    if (max_levels < 1 || max_levels > 23)
        return fail(VX_EINVAL, "vx_build_dense: max_levels must be in [1, 23]");
    auto* b = new (std::nothrow) vx_build();
    if (!b) return fail(VX_ENOMEM, "vx_build_dense: out of host memory");
    b->R = R;
    const uint32_t bpa = R / 8, wpr = R / 64;
    b->cfg.world_min[0] = b->cfg.world_min[1] = b->cfg.world_min[2] = 0.0f;
    b->cfg.world_max[0] = b->cfg.world_max[1] = b->cfg.world_max[2] = float(R);
    b->cfg.max_levels = max_levels;
    b->cfg.brick_depth = 3;
    b->cfg.bricks_per_axis = int32_t(bpa);

    // 1. per-slot occupancy masks (16 words) and populated flags, slab-parallel.
    const uint64_t slots = uint64_t(bpa) * bpa * bpa;
    std::vector<uint8_t> populated(slots, 0);
    parallel_for(int64_t(bpa), [&](int64_t bz) {
        for (uint32_t by = 0; by < bpa; ++by)
            for (uint32_t bx = 0; bx < bpa; ++bx) {
                uint8_t any = 0;
                for (uint32_t z = 0; z < 8 && !any; ++z)
                    for (uint32_t y = 0; y < 8; ++y) {
                        uint64_t w = (uint64_t(bz * 8 + z) * R + (by * 8 + y)) * wpr + (bx >> 3);
                        if ((bits[w] >> ((bx & 7) * 8)) & 0xFF) { any = 1; break; }
                    }
                populated[(uint64_t(bz) * bpa + by) * bpa + bx] = any;
            }
    });
    // 2. Morton order of populated bricks.
    std::vector<std::pair<uint64_t, uint32_t>> order;  // (morton, packed coord)
    for (uint64_t i = 0; i < slots; ++i)
        if (populated[i]) {
            uint32_t x = uint32_t(i % bpa), y = uint32_t((i / bpa) % bpa), z = uint32_t(i / (uint64_t(bpa) * bpa));
            order.push_back({morton3(x, y, z), x | (y << 10) | (z << 20)});
        }
    std::sort(order.begin(), order.end());
    const uint32_t B = uint32_t(order.size());
    b->coord.resize(B);
    b->occ.assign(size_t(B) * 16, 0u);
    b->grid.assign(slots, NONE);
    for (uint32_t i = 0; i < B; ++i) b->coord[i] = order[i].second;
    parallel_for(int64_t(B), [&](int64_t i) {
        uint32_t c = b->coord[size_t(i)];
        uint32_t bx = c & 0x3FF, by = (c >> 10) & 0x3FF, bz = (c >> 20) & 0x3FF;
        b->grid[(uint64_t(bz) * bpa + by) * bpa + bx] = uint32_t(i);
        uint32_t* w = &b->occ[size_t(i) * 16];
        for (uint32_t z = 0; z < 8; ++z)
            for (uint32_t y = 0; y < 8; ++y) {
                uint64_t wi = (uint64_t(bz * 8 + z) * R + (by * 8 + y)) * wpr + (bx >> 3);
                uint32_t row = uint32_t((bits[wi] >> ((bx & 7) * 8)) & 0xFF);
                w[z * 2 + (y >> 2)] |= row << ((y & 3) * 8);
            }
    });
    if (B == 0) { *out = b; return VX_OK; }  // empty octree (SVORebuild.cpp:358-361)

    // 3. Levels bottom-up (SVORebuild.cpp:446-518).  lvl[0] = bricks.
    struct Level { std::vector<uint32_t> coord; std::vector<uint8_t> valid; };
    std::vector<Level> lv(1);
    lv[0].coord = b->coord;
    const int brickDepth = 3;
    for (int depth = brickDepth + 1; depth <= max_levels; ++depth) {
        const Level& ch = lv.back();
        Level par;
        for (size_t i = 0; i < ch.coord.size(); ++i) {
            uint32_t c = ch.coord[i];
            uint32_t x = c & 0x3FF, y = (c >> 10) & 0x3FF, z = (c >> 20) & 0x3FF;
            uint32_t pc = (x >> 1) | ((y >> 1) << 10) | ((z >> 1) << 20);
            uint8_t oct = uint8_t((x & 1) | ((y & 1) << 1) | ((z & 1) << 2));
            if (par.coord.empty() || par.coord.back() != pc) {  // Morton order keeps siblings adjacent
                par.coord.push_back(pc);
                par.valid.push_back(0);
            }
            par.valid.back() |= uint8_t(1u << oct);
        }
        bool isRoot = par.coord.size() == 1 && par.coord[0] == 0;
        lv.push_back(std::move(par));
        if (isRoot) break;
    }
    if (lv.back().coord.size() != 1) {
        delete b;
        return fail(VX_EINVAL, "vx_build_dense: several nodes at the top level (max_levels too small for R)");
    }
    // 4. Layout: top level first.
    const int L = int(lv.size());
    std::vector<uint32_t> off(size_t(L) + 1, 0);  // off[k] for level index from the top
    for (int k = 0; k < L; ++k) off[size_t(k) + 1] = off[size_t(k)] + uint32_t(lv[size_t(L - 1 - k)].coord.size());
    const uint32_t D = off[size_t(L)];
    b->nodes.resize(D);
    b->node_brick.assign(D, 0u);
    for (int k = 0; k < L; ++k) {
        const Level& lev = lv[size_t(L - 1 - k)];
        const bool bricks = (k == L - 1);
        uint32_t next = off[size_t(k) + 1];
        for (size_t i = 0; i < lev.coord.size(); ++i) {
            vx_node& nd = b->nodes[off[size_t(k)] + i];
            if (bricks) {
                nd.child_ptr = 0;
                nd.masks = 0xFFu | (0xFFu << 8);
                b->node_brick[off[size_t(k)] + i] = uint32_t(i);
            } else {
                uint8_t v = lev.valid[i];
                uint8_t leaf = (k == L - 2) ? v : 0;  // children are bricks
                nd.child_ptr = next;
                nd.masks = uint32_t(v) | (uint32_t(leaf) << 8);
                next += uint32_t(__builtin_popcount(v));
            }
        }
    }
    *out = b;
    return VX_OK;
}

int vx_build_dense(const uint64_t* bits, uint32_t R, int32_t max_levels, vx_build** out) {
    return vx::guarded("vx_build_dense", [&] { return vx_build_dense_body(bits, R, max_levels, out); });
}

int vx_build_desc(const vx_build* b, vx_scene_desc* d) {
    using namespace vx;
    if (!b || !d) return fail(VX_EINVAL, "vx_build_desc: null argument");
    std::memset(d, 0, sizeof(*d));
    d->config = b->cfg;
    d->nodes = b->nodes.data();
    d->node_count = uint32_t(b->nodes.size());
    d->brick_count = uint32_t(b->coord.size());
    d->node_brick = b->node_brick.data();
    d->grid_lookup = b->grid.data();
    d->brick_coord = b->coord.data();
    d->brick_occ = b->occ.data();
    d->color_kind = VX_COLOR_NONE;
    d->brick_color = nullptr;
    return VX_OK;
}

int vx_build_free(vx_build* b) {
    delete b;
    return VX_OK;
}

int vx_nodes_from_reference(const uint64_t* ref, uint32_t n, vx_node* nodes, uint32_t* node_brick) {
    using namespace vx;
    if ((!ref && n) || (!nodes && n)) return fail(VX_EINVAL, "vx_nodes_from_reference: null argument");
    for (uint32_t i = 0; i < n; ++i) {
        // ChildDescriptor bit-fields, first field in the least significant
        // bits (SVOTypes.h:38-46, GCC/Clang/MSVC little-endian layout).
        uint64_t v = ref[i];
        uint32_t lo = uint32_t(v), hi = uint32_t(v >> 32);
        uint32_t cp = lo & 0x7FFF, far = (lo >> 15) & 1, valid = (lo >> 16) & 0xFF, leaf = (lo >> 24) & 0xFF;
        if (far) return fail(VX_EINVAL, "vx_nodes_from_reference: far pointers are not supported");
        nodes[i].child_ptr = cp;
        nodes[i].masks = valid | (leaf << 8);
        if (node_brick) node_brick[i] = hi & 0xFFFFFF;
    }
    return VX_OK;
}

// ---------------------------------------------------------------------------
// Synthetic inputs
// ---------------------------------------------------------------------------

// Value noise.  Lattice value of octave o at integer lattice point (i,j,k):
// (hash >> 40) * 2^-24.  Voxel (x,y,z) samples p = (x + 0.5) / s_o with
// s_o = spacing >> o, f = p - floor(p), w = f*f*(3 - 2f); the cell is blended
// along y, then z, then x; octaves are summed with weight 0.5^o in order.
static int vx_synth_noise_body(uint32_t R, uint32_t spacing, uint32_t octaves, float fill, uint64_t seed, int32_t shell,
                   uint64_t* out_bits) {
    using namespace vx;
    if (!out_bits || R < 64 || R % 64 != 0 || R > 4096 || octaves < 1 || octaves > 16 || spacing < 1 ||
        (spacing >> (octaves - 1)) < 1 || !(fill >= 0.0f && fill <= 1.0f))
        return fail(VX_EINVAL, "vx_synth_noise: bad arguments");
    const uint64_t N = uint64_t(R) * R * R;
    std::vector<float> field;
    try { field.resize(N); } catch (...) { return fail(VX_ENOMEM, "vx_synth_noise: out of host memory"); }
    struct Oct { uint32_t s; float inv_s, amp; uint32_t cells; std::vector<float> lat; };
    std::vector<Oct> oc(octaves);
    float amp = 1.0f;
    for (uint32_t o = 0; o < octaves; ++o) {
        oc[o].s = spacing >> o;
        oc[o].amp = amp;
        amp *= 0.5f;
        oc[o].cells = (R + oc[o].s - 1) / oc[o].s + 2;
    }
    // Lattice tables (cells^3 per octave), hashed once.
    for (uint32_t o = 0; o < octaves; ++o) {
        const uint32_t c = oc[o].cells;
        oc[o].lat.resize(size_t(c) * c * c);
        float* lat = oc[o].lat.data();
        parallel_for(int64_t(c), [&, o, c, lat](int64_t k) {
            for (uint32_t j = 0; j < c; ++j)
                for (uint32_t i = 0; i < c; ++i)
                    lat[(size_t(k) * c + j) * c + i] =
                        float(hash4(seed, o, i, j, uint32_t(k)) >> 40) * (1.0f / 16777216.0f);
        });
    }
    // Field, one (y,z) row at a time.
    parallel_for(int64_t(R) * R, [&](int64_t row) {
        const uint32_t y = uint32_t(row % R), z = uint32_t(row / R);
        float* out = &field[size_t(row) * R];
        std::vector<float> lz;
        for (uint32_t x = 0; x < R; ++x) out[x] = 0.0f;
        for (uint32_t o = 0; o < octaves; ++o) {
            const Oct& q = oc[o];
            const float fs = float(q.s);
            float py = (float(y) + 0.5f) / fs, pz = (float(z) + 0.5f) / fs;
            float jy = std::floor(py), kz = std::floor(pz);
            float fy = py - jy, fz = pz - kz;
            float wy = fy * fy * (3.0f - 2.0f * fy), wz = fz * fz * (3.0f - 2.0f * fz);
            uint32_t j = uint32_t(jy), k = uint32_t(kz);
            const uint32_t c = q.cells;
            const uint32_t ni = R / q.s + 2;
            lz.resize(ni);
            for (uint32_t i = 0; i < ni; ++i) {
                const float* l = q.lat.data();
                float a0 = l[(size_t(k) * c + j) * c + i], b0 = l[(size_t(k) * c + j + 1) * c + i];
                float a1 = l[(size_t(k + 1) * c + j) * c + i], b1 = l[(size_t(k + 1) * c + j + 1) * c + i];
                float ly0 = a0 + wy * (b0 - a0);
                float ly1 = a1 + wy * (b1 - a1);
                lz[i] = ly0 + wz * (ly1 - ly0);
            }
            for (uint32_t x = 0; x < R; ++x) {
                float px = (float(x) + 0.5f) / fs;
                float ix = std::floor(px);
                float fx = px - ix;
                float wx = fx * fx * (3.0f - 2.0f * fx);
                uint32_t i = uint32_t(ix);
                float v = lz[i] + wx * (lz[i + 1] - lz[i]);
                out[x] = out[x] + q.amp * v;
            }
        }
    });
    // Threshold: the value of ascending rank N - n_solid (radix select on the
    // bit patterns of the non-negative values); solid = value >= threshold.
    const uint64_t n_solid = uint64_t(std::floor(double(fill) * double(N) + 0.5));
    uint32_t thr_bits = 0xFFFFFFFFu;  // nothing solid
    if (n_solid > 0) {
        const uint64_t rank = N - n_solid;  // 0-based ascending rank
        const int T = hw_threads();
        auto histo = [&](int shift, uint32_t prefix_mask, uint32_t prefix, std::vector<uint64_t>& h) {
            std::vector<std::vector<uint64_t>> loc(size_t(T), std::vector<uint64_t>(65536, 0));
            std::atomic<int> tid{0};
            const int64_t chunks = 4096;
            std::vector<std::thread> th;
            std::atomic<int64_t> next{0};
            for (int t = 0; t < T; ++t)
                th.emplace_back([&] {
                    std::vector<uint64_t>& mine = loc[size_t(tid.fetch_add(1))];
                    for (int64_t ci; (ci = next.fetch_add(1)) < chunks;) {
                        uint64_t b0 = N * uint64_t(ci) / chunks, b1 = N * uint64_t(ci + 1) / chunks;
                        for (uint64_t i = b0; i < b1; ++i) {
                            uint32_t u;
                            std::memcpy(&u, &field[i], 4);
                            if ((u & prefix_mask) == prefix) mine[(u >> shift) & 0xFFFF]++;
                        }
                    }
                });
            for (auto& x : th) x.join();
            h.assign(65536, 0);
            for (auto& l : loc)
                for (int i = 0; i < 65536; ++i) h[size_t(i)] += l[size_t(i)];
        };
        std::vector<uint64_t> h;
        histo(16, 0, 0, h);
        uint64_t acc = 0, r = rank;
        uint32_t hi = 0;
        for (uint32_t i = 0; i < 65536; ++i) {
            if (acc + h[i] > r) { hi = i; r -= acc; break; }
            acc += h[i];
        }
        histo(0, 0xFFFF0000u, hi << 16, h);
        acc = 0;
        uint32_t lo = 0;
        for (uint32_t i = 0; i < 65536; ++i) {
            if (acc + h[i] > r) { lo = i; break; }
            acc += h[i];
        }
        thr_bits = (hi << 16) | lo;
    }
    float thr;
    std::memcpy(&thr, &thr_bits, 4);
    const uint32_t wpr = R / 64;
    parallel_for(int64_t(R) * R, [&](int64_t row) {
        const uint32_t y = uint32_t(row % R), z = uint32_t(row / R);
        const float* f = &field[size_t(row) * R];
        for (uint32_t w = 0; w < wpr; ++w) {
            uint64_t word = 0;
            for (uint32_t bit = 0; bit < 64; ++bit) {
                uint32_t x = w * 64 + bit;
                bool solid = (n_solid > 0) && f[x] >= thr;
                if (shell && (x == 0 || y == 0 || z == 0 || x == R - 1 || y == R - 1 || z == R - 1)) solid = true;
                word |= uint64_t(solid) << bit;
            }
            out_bits[size_t(row) * wpr + w] = word;
        }
    });
    return VX_OK;
}

int vx_synth_noise(uint32_t R, uint32_t spacing, uint32_t octaves, float fill, uint64_t seed, int32_t shell,
                   uint64_t* out_bits) {
    return vx::guarded("vx_synth_noise", [&] { return vx_synth_noise_body(R, spacing, octaves, fill, seed, shell, out_bits); });
}

static int vx_synth_urban_body(uint32_t R, uint32_t hmin, uint32_t hmax, uint64_t seed, uint64_t* out_bits) {
    using namespace vx;
    if (!out_bits || R < 64 || R % 64 != 0 || R > 8192 || hmin > hmax)
        return fail(VX_EINVAL, "vx_synth_urban: bad arguments");
    // 32 x 32 blocks; streets 8 voxels wide at R = 2048, scaled with R (at least 1).
    const uint32_t pitch = R / 32, street = std::max(1u, R / 256), block = pitch - street, wpr = R / 64;
    uint32_t height[32][32];
    for (uint32_t bz = 0; bz < 32; ++bz)
        for (uint32_t bx = 0; bx < 32; ++bx) {
            uint64_t h = hash4(seed, 0x75726Bu, bx, bz, 0);
            uint32_t v = hmin + uint32_t(h % uint64_t(hmax - hmin + 1));
            height[bz][bx] = std::min(v, R);
        }
    parallel_for(int64_t(R) * R, [&](int64_t row) {
        const uint32_t y = uint32_t(row % R), z = uint32_t(row / R);
        const uint32_t bz = z / pitch, lzz = z % pitch;
        for (uint32_t w = 0; w < wpr; ++w) {
            uint64_t word = 0;
            for (uint32_t bit = 0; bit < 64; ++bit) {
                uint32_t x = w * 64 + bit;
                uint32_t bx = x / pitch, lxx = x % pitch;
                bool solid = lxx < block && lzz < block && y < height[bz][bx];
                word |= uint64_t(solid) << bit;
            }
            out_bits[size_t(row) * wpr + w] = word;
        }
    });
    return VX_OK;
}

int vx_synth_urban(uint32_t R, uint32_t hmin, uint32_t hmax, uint64_t seed, uint64_t* out_bits) {
    return vx::guarded("vx_synth_urban", [&] { return vx_synth_urban_body(R, hmin, hmax, seed, out_bits); });
}

static int vx_synth_rgba8_body(const uint32_t* coord, uint32_t B, uint64_t seed, uint32_t* out) {
    using namespace vx;
    if ((!coord || !out) && B) return fail(VX_EINVAL, "vx_synth_rgba8: null argument");
    parallel_for(int64_t(B), [&](int64_t b) {
        for (uint32_t v = 0; v < 512; ++v)
            out[size_t(b) * 512 + v] = vx::synth_rgba8_word(seed, coord[b], v);
    });
    return VX_OK;
}

int vx_synth_rgba8(const uint32_t* coord, uint32_t B, uint64_t seed, uint32_t* out) {
    return vx::guarded("vx_synth_rgba8", [&] { return vx_synth_rgba8_body(coord, B, seed, out); });
}

static int vx_synth_dxt1_body(const uint32_t* coord, uint32_t B, uint64_t seed, uint64_t* out) {
    using namespace vx;
    if ((!coord || !out) && B) return fail(VX_EINVAL, "vx_synth_dxt1: null argument");
    parallel_for(int64_t(B), [&](int64_t b) {
        for (uint32_t k = 0; k < 32; ++k) out[size_t(b) * 32 + k] = vx::synth_dxt1_block(seed, coord[b], k);
    });
    return VX_OK;
}

int vx_synth_dxt1(const uint32_t* coord, uint32_t B, uint64_t seed, uint64_t* out) {
    return vx::guarded("vx_synth_dxt1", [&] { return vx_synth_dxt1_body(coord, B, seed, out); });
}

}  // extern "C"
