// vx_gpubuild.cu - the scene builder on the device: the arrays of
// vx_build_dense (vx_build.cpp), index for index, from occupancy bits already
// in device memory, written straight into a new scene's pool.
//
// vx_build_dense's closed form of LaineKarrasOctree::rebuild
// (SVO/src/SVORebuild.cpp:228-607): brick index = rank of the brick's grid
// coordinate in Morton order; descriptors top level first, each level in
// Morton order of its node coordinates; a node's child pointer = offset of the
// level below + the Morton rank of its first child there.  On the device every
// level is a flag array over the Morton cells of that level (the brick level
// has P^3 cells, P = bricks per axis rounded up to a power of two, each level
// above 8 times fewer), and every rank is an exclusive prefix sum of flags:
//   e_0[m]  = brick at Morton code m holds a voxel
//   e_j[c]  = any of e_{j-1}[8c .. 8c+7];  valid_j[c] = those 8 flags as a mask
//   rank_j  = exclusive scan of e_j
// The climb stops like the host builder's: at the first level whose only node
// is the cell at coordinate 0 (the root), or at depth max_levels.
#include <algorithm>
#include <vector>

#include "vx_hash.h"
#include "vx_internal.h"

extern "C" int vx_build_normals_dev(const uint32_t* occ_dev, uint32_t brick_count, uint64_t* out_dev, void* stream);

namespace vx {
namespace {

constexpr uint32_t NONE_ = 0xFFFFFFFFu;

// ---- exclusive prefix sum of u32 (reduce, scan the tile sums, rescan) ----
constexpr int SCAN_T = 256;
constexpr int SCAN_I = 16;
constexpr uint64_t SCAN_TILE = uint64_t(SCAN_T) * SCAN_I;

// Exclusive scan of v over the block; *total gets the block sum.
__device__ __forceinline__ uint32_t block_exclusive(uint32_t v, uint32_t& total) {
    __shared__ uint32_t warp_sums[SCAN_T / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < SCAN_T / 32 ? warp_sums[lane] : 0u;
#pragma unroll
        for (int o = 1; o < SCAN_T / 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < SCAN_T / 32) warp_sums[lane] = w;
    }
    __syncthreads();
    total = warp_sums[SCAN_T / 32 - 1];
    return (warp ? warp_sums[warp - 1] : 0u) + x - v;
}

__global__ void __launch_bounds__(SCAN_T) tile_reduce_kernel(const uint32_t* __restrict__ in, uint64_t n,
                                                             uint32_t* __restrict__ sums) {
    const uint64_t base = uint64_t(blockIdx.x) * SCAN_TILE;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_I; ++k) {
        const uint64_t i = base + uint64_t(k) * SCAN_T + threadIdx.x;
        if (i < n) s += in[i];
    }
    uint32_t total;
    block_exclusive(s, total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// out[i] = offs[tile] + exclusive sum within the tile; *total = sum of all.
__global__ void __launch_bounds__(SCAN_T) tile_scan_kernel(const uint32_t* __restrict__ in, uint64_t n,
                                                           const uint32_t* __restrict__ offs,
                                                           uint32_t* __restrict__ out, uint32_t* __restrict__ total) {
    const uint64_t base = uint64_t(blockIdx.x) * SCAN_TILE + uint64_t(threadIdx.x) * SCAN_I;
    uint32_t v[SCAN_I];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_I; ++k) {
        v[k] = (base + k < n) ? in[base + k] : 0u;
        s += v[k];
    }
    uint32_t bt;
    uint32_t run = block_exclusive(s, bt) + (offs ? offs[blockIdx.x] : 0u);
#pragma unroll
    for (int k = 0; k < SCAN_I; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
    if (total && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *total = (offs ? offs[blockIdx.x] : 0u) + bt;
}

uint64_t scan_scratch_words(uint64_t n) {
    const uint64_t t = (n + SCAN_TILE - 1) / SCAN_TILE;
    return t <= 1 ? 0 : 2 * t + scan_scratch_words(t);
}

void exclusive_scan(const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* total, uint32_t* scratch,
                    cudaStream_t st) {
    const uint64_t t = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (t <= 1) {
        tile_scan_kernel<<<1, SCAN_T, 0, st>>>(in, n, nullptr, out, total);
        return;
    }
    uint32_t* sums = scratch;
    uint32_t* offs = scratch + t;
    tile_reduce_kernel<<<uint32_t(t), SCAN_T, 0, st>>>(in, n, sums);
    exclusive_scan(sums, offs, t, nullptr, scratch + 2 * t, st);
    tile_scan_kernel<<<uint32_t(t), SCAN_T, 0, st>>>(in, n, offs, out, total);
}

// ---- brick level ----
struct BitGrid {
    const uint8_t* bytes;  // occupancy bits as bytes: byte (z * R + y) * (R / 8) + bx holds x = 8 bx .. 8 bx + 7
    uint32_t R, bpa;
};

__device__ __forceinline__ uint8_t row_byte(const BitGrid& g, uint32_t bx, uint32_t y, uint32_t z) {
    return __ldg(g.bytes + (uint64_t(z) * g.R + y) * (g.R / 8) + bx);
}

// e_0[morton(slot)] = slot holds a voxel.  One thread per slot in linear order
// (x fastest), so a warp's row reads are 32 adjacent bytes.
__global__ void __launch_bounds__(256) brick_flags_kernel(BitGrid g, uint32_t* __restrict__ e0) {
    const uint64_t slots = uint64_t(g.bpa) * g.bpa * g.bpa;
    for (uint64_t s = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; s < slots;
         s += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t bx = uint32_t(s % g.bpa), by = uint32_t((s / g.bpa) % g.bpa),
                       bz = uint32_t(s / (uint64_t(g.bpa) * g.bpa));
        uint32_t any = 0;
        for (uint32_t z = 0; z < 8; ++z)
#pragma unroll
            for (uint32_t y = 0; y < 8; ++y) any |= row_byte(g, bx, by * 8 + y, bz * 8 + z);
        if (any) e0[morton3(bx, by, bz)] = 1u;
    }
}

// brickGridLookup, brick coordinates and occupancy words of every slot.
__global__ void __launch_bounds__(256) brick_scatter_kernel(BitGrid g, const uint32_t* __restrict__ rank0,
                                                            uint32_t* __restrict__ grid, uint32_t* __restrict__ coord,
                                                            uint4* __restrict__ occ) {
    const uint64_t slots = uint64_t(g.bpa) * g.bpa * g.bpa;
    for (uint64_t s = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; s < slots;
         s += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t bx = uint32_t(s % g.bpa), by = uint32_t((s / g.bpa) % g.bpa),
                       bz = uint32_t(s / (uint64_t(g.bpa) * g.bpa));
        uint32_t w[16];
        uint32_t any = 0;
#pragma unroll
        for (int k = 0; k < 16; ++k) w[k] = 0;
#pragma unroll
        for (uint32_t z = 0; z < 8; ++z)
#pragma unroll
            for (uint32_t y = 0; y < 8; ++y) {
                const uint32_t row = row_byte(g, bx, by * 8 + y, bz * 8 + z);
                any |= row;
                w[z * 2 + (y >> 2)] |= row << ((y & 3) * 8);  // voxel z*64 + y*8 + x: word >> 5, bit & 31
            }
        if (!any) {
            grid[s] = NONE_;
            continue;
        }
        const uint32_t b = rank0[morton3(bx, by, bz)];
        grid[s] = b;
        coord[b] = bx | (by << 10) | (bz << 20);
        uint4* o = occ + uint64_t(b) * 4;
#pragma unroll
        for (int k = 0; k < 4; ++k) o[k] = make_uint4(w[4 * k], w[4 * k + 1], w[4 * k + 2], w[4 * k + 3]);
    }
}

// ---- levels above the bricks ----
__global__ void __launch_bounds__(256) level_kernel(const uint32_t* __restrict__ below, uint64_t cells,
                                                    uint32_t* __restrict__ e, uint8_t* __restrict__ valid) {
    for (uint64_t c = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; c < cells;
         c += uint64_t(gridDim.x) * blockDim.x) {
        const uint4 a = reinterpret_cast<const uint4*>(below)[2 * c];
        const uint4 b = reinterpret_cast<const uint4*>(below)[2 * c + 1];
        const uint32_t v = (a.x ? 1u : 0u) | (a.y ? 2u : 0u) | (a.z ? 4u : 0u) | (a.w ? 8u : 0u) | (b.x ? 16u : 0u) |
                           (b.y ? 32u : 0u) | (b.z ? 64u : 0u) | (b.w ? 128u : 0u);
        e[c] = v ? 1u : 0u;
        valid[c] = uint8_t(v);
    }
}

// Descriptors of one level.  Bricks: child pointer 0, valid = leaf = 0xFF and
// the brick index (SVORebuild.cpp:419-443); the level above the bricks has
// leaf = valid, the rest leaf = 0.
__global__ void __launch_bounds__(256) nodes_kernel(const uint32_t* __restrict__ e, const uint32_t* __restrict__ rank,
                                                    const uint8_t* __restrict__ valid,
                                                    const uint32_t* __restrict__ rank_below, uint64_t cells,
                                                    uint32_t off, uint32_t off_below, int is_bricks,
                                                    int children_are_bricks, uint2* __restrict__ nodes,
                                                    uint32_t* __restrict__ node_brick) {
    for (uint64_t c = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; c < cells;
         c += uint64_t(gridDim.x) * blockDim.x) {
        if (!e[c]) continue;
        const uint32_t r = rank[c], idx = off + r;
        if (is_bricks) {
            nodes[idx] = make_uint2(0u, 0xFFFFu);
            node_brick[idx] = r;
        } else {
            const uint32_t v = valid[c];
            nodes[idx] = make_uint2(off_below + rank_below[8 * c], v | (children_are_bricks ? v << 8 : 0u));
            node_brick[idx] = 0u;
        }
    }
}

// ---- colour payloads (vx_synth_rgba8 / vx_synth_dxt1) ----
__global__ void __launch_bounds__(256) rgba8_kernel(const uint32_t* __restrict__ coord, uint64_t words, uint64_t seed,
                                                    uint32_t* __restrict__ out) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < words;
         i += uint64_t(gridDim.x) * blockDim.x)
        out[i] = synth_rgba8_word(seed, __ldg(coord + (i >> 9)), uint32_t(i & 511));
}
__global__ void __launch_bounds__(256) dxt1_kernel(const uint32_t* __restrict__ coord, uint64_t blocks, uint64_t seed,
                                                   uint64_t* __restrict__ out) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < blocks;
         i += uint64_t(gridDim.x) * blockDim.x)
        out[i] = synth_dxt1_block(seed, __ldg(coord + (i >> 5)), uint32_t(i & 31));
}

uint32_t grid_for(uint64_t n, int sms) {
    return uint32_t(std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, uint64_t(sms) * 32)));
}

int cerr(cudaError_t e, const char* what) {
    return fail(VX_ECUDA, std::string("vx_scene_create_dense_dev: ") + what + ": " + cudaGetErrorName(e) + " (" +
                              cudaGetErrorString(e) + ")");
}

}  // namespace
}  // namespace vx

static int vx_scene_create_dense_dev_body(const uint64_t* bits_dev, uint32_t R, int32_t max_levels, int32_t color_kind,
                                         uint64_t color_seed, int32_t with_normals, vx_scene** out, void* stream) {
    using namespace vx;
    if (!bits_dev || !out) return fail(VX_EINVAL, "vx_scene_create_dense_dev: null argument");
    *out = nullptr;
    if (R < 64 || R % 64 != 0 || R > 4096)
        return fail(VX_EINVAL, "vx_scene_create_dense_dev: R must be a multiple of 64 in [64, 4096]");
    if (max_levels < 1 || max_levels > 23)
        return fail(VX_EINVAL, "vx_scene_create_dense_dev: max_levels must be in [1, 23]");
    if (color_kind != VX_COLOR_NONE && color_kind != VX_COLOR_RGBA8 && color_kind != VX_COLOR_DXT1)
        return fail(VX_EINVAL, "vx_scene_create_dense_dev: unknown color_kind");
    if (reinterpret_cast<uintptr_t>(bits_dev) % 8) return fail(VX_EINVAL, "vx_scene_create_dense_dev: misaligned bits");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);

    const uint32_t bpa = R / 8;
    uint32_t P = 1, logP = 0;
    while (P < bpa) { P <<= 1; ++logP; }
    // level j has N_j = P^3 / 8^j cells, j = 0 .. logP
    std::vector<uint64_t> N(logP + 1), at(logP + 2, 0), vat(logP + 2, 0);
    for (uint32_t j = 0; j <= logP; ++j) {
        N[j] = uint64_t(1) << (3 * (logP - j));
        at[j + 1] = at[j] + ((N[j] + 3) & ~uint64_t(3));  // keep every level 16-byte aligned
        vat[j + 1] = vat[j] + ((N[j] + 15) & ~uint64_t(15));
    }
    const uint64_t flag_words = at[logP + 1], scratch_words = scan_scratch_words(N[0]) + 64;
    const uint64_t tmp_bytes = (2 * flag_words + scratch_words) * 4 + vat[logP + 1];
    char* tmp = nullptr;
    cudaError_t e = cudaMalloc(&tmp, tmp_bytes);
    if (e != cudaSuccess) return cerr(e, "cudaMalloc scratch");
    uint32_t* E = reinterpret_cast<uint32_t*>(tmp);
    uint32_t* RK = E + flag_words;
    uint32_t* scratch = RK + flag_words;
    uint32_t* counts = scratch + scratch_words - 64;  // counts[j]: nodes in level j
    uint8_t* V = reinterpret_cast<uint8_t*>(scratch + scratch_words);
    auto done = [&](int r) {
        cudaFree(tmp);
        return r;
    };
    const BitGrid g{reinterpret_cast<const uint8_t*>(bits_dev), R, bpa};
    const uint64_t slots = uint64_t(bpa) * bpa * bpa;

    // brick level
    e = cudaMemsetAsync(E, 0, N[0] * 4, st);
    if (e != cudaSuccess) return done(cerr(e, "memset"));
    brick_flags_kernel<<<grid_for(slots, sms), 256, 0, st>>>(g, E);
    exclusive_scan(E, RK, N[0], counts, scratch, st);
    uint32_t B = 0;
    e = cudaMemcpyAsync(&B, counts, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return done(cerr(e, "brick level"));

    // levels above, bottom-up (SVORebuild.cpp:446-518)
    std::vector<uint32_t> n_at{B};
    uint32_t top = 0;  // highest level built
    if (B > 0) {
        for (int depth = 4; depth <= max_levels && top < logP; ++depth) {
            const uint32_t j = top + 1;
            level_kernel<<<grid_for(N[j], sms), 256, 0, st>>>(E + at[j - 1], N[j], E + at[j], V + vat[j]);
            exclusive_scan(E + at[j], RK + at[j], N[j], counts + j, scratch, st);
            uint32_t info[2] = {0, 0};
            e = cudaMemcpyAsync(&info[0], counts + j, 4, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(&info[1], E + at[j], 4, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return done(cerr(e, "level"));
            n_at.push_back(info[0]);
            top = j;
            if (info[0] == 1 && info[1] == 1) break;  // the only node is at coordinate 0: the root
        }
        if (n_at.back() != 1)
            return done(fail(VX_EINVAL, "vx_scene_create_dense_dev: several nodes at the top level (max_levels too "
                                        "small for R)"));
    }
    // layout: top level first
    const uint32_t L = B ? top + 1 : 0;
    std::vector<uint32_t> off(L + 1, 0);  // off[k], k = 0 the top level
    for (uint32_t k = 0; k < L; ++k) off[k + 1] = off[k] + n_at[L - 1 - k];
    const uint32_t D = L ? off[L] : 0;

    vx_octree_config cfg{};
    cfg.world_max[0] = cfg.world_max[1] = cfg.world_max[2] = float(R);
    cfg.max_levels = max_levels;
    cfg.brick_depth = 3;
    cfg.bricks_per_axis = int32_t(bpa);
    vx_scene* scene = nullptr;
    ScenePool p{};
    if (int r = scene_alloc(cfg, D, B, color_kind, with_normals != 0 && B > 0, &scene, &p)) return done(r);
    uint32_t* grid = static_cast<uint32_t*>(p.grid);
    brick_scatter_kernel<<<grid_for(slots, sms), 256, 0, st>>>(g, RK, grid, static_cast<uint32_t*>(p.coord),
                                                               static_cast<uint4*>(p.occ));
    for (uint32_t j = 0; j < L; ++j) {
        const uint32_t k = L - 1 - j;
        nodes_kernel<<<grid_for(N[j], sms), 256, 0, st>>>(
            E + at[j], RK + at[j], j ? V + vat[j] : nullptr, j ? RK + at[j - 1] : nullptr, N[j], off[k],
            k + 1 <= L - 1 ? off[k + 1] : 0u, j == 0, j == 1, static_cast<uint2*>(p.nodes),
            static_cast<uint32_t*>(p.node_brick));
    }
    if (color_kind == VX_COLOR_RGBA8 && B)
        rgba8_kernel<<<grid_for(uint64_t(B) * 512, sms), 256, 0, st>>>(static_cast<const uint32_t*>(p.coord),
                                                                       uint64_t(B) * 512, color_seed,
                                                                       static_cast<uint32_t*>(p.color));
    if (color_kind == VX_COLOR_DXT1 && B)
        dxt1_kernel<<<grid_for(uint64_t(B) * 32, sms), 256, 0, st>>>(static_cast<const uint32_t*>(p.coord),
                                                                     uint64_t(B) * 32, color_seed,
                                                                     static_cast<uint64_t*>(p.color));
    e = cudaGetLastError();
    if (e != cudaSuccess) { vx_scene_destroy(scene); return done(cerr(e, "launch")); }
    if (p.nrm) {
        if (int r = vx_build_normals_dev(static_cast<const uint32_t*>(p.occ), B, static_cast<uint64_t*>(p.nrm), stream)) {
            vx_scene_destroy(scene);
            return done(r);
        }
    }
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { vx_scene_destroy(scene); return done(cerr(e, "synchronize")); }
    *out = scene;
    return done(VX_OK);
}

extern "C" int vx_scene_create_dense_dev(const uint64_t* bits_dev, uint32_t R, int32_t max_levels, int32_t color_kind,
                                         uint64_t color_seed, int32_t with_normals, vx_scene** out, void* stream) {
    return vx::guarded("vx_scene_create_dense_dev", [&] { return vx_scene_create_dense_dev_body(bits_dev, R, max_levels, color_kind, color_seed, with_normals, out, stream); });
}
