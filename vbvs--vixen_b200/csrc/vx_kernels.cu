// vx_kernels.cu - plain (one launch per scene) cast and render kernels.
#include "vx_cast.cuh"
#include "vx_palette.h"

namespace vx {
namespace {

// Threads per block of the cast kernel, and warps per block of the render
// kernel (each warp one 8 x 4 piece of a 32 x 8 tile).
#ifndef VX_CAST_BLOCK
#define VX_CAST_BLOCK 64
#endif
#ifndef VX_RENDER_WARPS
#define VX_RENDER_WARPS 2
#endif
constexpr int BLOCK = VX_CAST_BLOCK;
constexpr int RENDER_WARPS = VX_RENDER_WARPS;
constexpr int RENDER_THREADS = RENDER_WARPS * 32;
// Resident blocks per SM the cast kernel is compiled for: 14 blocks of 64
// threads leave 72 registers a thread (cfg2 frame 0.1208 -> 0.1188 ms against
// 12 blocks at 80 registers; 16 blocks at 64 registers spill and measure
// 0.1249 ms).
constexpr int CAST_MIN_BLOCKS = 896 / BLOCK;

template <bool LOD>
__global__ void __launch_bounds__(BLOCK, CAST_MIN_BLOCKS) cast_kernel(DevScene s, const vx_ray* __restrict__ rays, uint32_t n,
                                                      float tmin, float tmax, vx_hit* __restrict__ hits,
                                                      void* __restrict__ color,
                                                      vx_ray_counters* __restrict__ counters, LodCone lod) {
    extern __shared__ uint32_t smem[];
    uint32_t* stkN = smem + threadIdx.x;
    float* stkT = reinterpret_cast<float*>(smem + s.max_levels * BLOCK) + threadIdx.x;
    uint32_t* cyc = smem + 2 * s.max_levels * BLOCK + threadIdx.x;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float2* r2 = reinterpret_cast<const float2*>(rays + i);
    const float2 a = __ldg(r2), b = __ldg(r2 + 1), c = __ldg(r2 + 2);
    Hit h;
    cast_ray<LOD>(s, a.x, a.y, b.x, b.y, c.x, c.y, tmin, tmax, stkN, stkT, cyc, BLOCK, h, lod);
    store_hit(hits, i, h);
    if (color) store_color(s, color, i, h);
    if (counters) {
        uint4 rc;
        rc.x = (h.iters & 0xFFFFu) | (h.grid_reads << 16);
        rc.y = h.dda_steps;
        rc.z = (h.run_iters & 0xFFFFu) | (h.run_grid_reads << 16);
        rc.w = h.run_dda_steps;
        reinterpret_cast<uint4*>(counters)[i] = rc;
    }
}

// The cast of rays compacted on the device: `count` (device) rays of at most
// n_max, the hit record of ray i going to slot map[i].  The per-ray work is
// cast_kernel's (castRay, no colour or counters).
__global__ void __launch_bounds__(BLOCK, 768 / BLOCK) cast_mapped_kernel(DevScene s, const vx_ray* __restrict__ rays,
                                                                        uint32_t n_max, const uint32_t* __restrict__ count,
                                                                        const uint32_t* __restrict__ map, float tmin,
                                                                        float tmax, vx_hit* __restrict__ hits) {
    extern __shared__ uint32_t smem[];
    uint32_t* stkN = smem + threadIdx.x;
    float* stkT = reinterpret_cast<float*>(smem + s.max_levels * BLOCK) + threadIdx.x;
    uint32_t* cyc = smem + 2 * s.max_levels * BLOCK + threadIdx.x;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= min(n_max, __ldg(count))) return;
    const float2* r2 = reinterpret_cast<const float2*>(rays + i);
    const float2 a = __ldg(r2), b = __ldg(r2 + 1), c = __ldg(r2 + 2);
    Hit h;
    cast_ray(s, a.x, a.y, b.x, b.y, c.x, c.y, tmin, tmax, stkN, stkT, cyc, BLOCK, h);
    store_hit(hits, __ldg(map + i), h);
}

// Pixels go to warps in 8 x 4 pieces of 32 x 8 tiles (the reference dispatches
// 8 x 8 workgroups, ComputeDispatchNode.cpp:272-301): a warp's rays are
// neighbours in both image directions, so their traversals diverge less than
// along a row.  Warp task t is piece t & 7 of tile t >> 3; a block holds
// RENDER_WARPS consecutive tasks.  Outputs are indexed by pixel (y * w + x).
__global__ void __launch_bounds__(RENDER_THREADS, 768 / RENDER_THREADS) render_kernel(
    DevScene s, CameraDev cam, uint32_t w, uint32_t hgt, uint32_t* __restrict__ image, vx_hit* __restrict__ hits,
    void* __restrict__ color) {
    extern __shared__ uint32_t smem[];
    uint32_t* stkN = smem + threadIdx.x;
    float* stkT = reinterpret_cast<float*>(smem + s.max_levels * RENDER_THREADS) + threadIdx.x;
    uint32_t* cyc = smem + 2 * s.max_levels * RENDER_THREADS + threadIdx.x;
    const uint32_t tw = (w + 31) / 32;
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t t = uint64_t(blockIdx.x) * RENDER_WARPS + (threadIdx.x >> 5);
    const uint32_t piece = uint32_t(t & 7u), tile = uint32_t(t >> 3);
    const uint32_t px = (tile % tw) * 32 + (piece & 3u) * 8 + (lane & 7u);
    const uint32_t py = (tile / tw) * 8 + (piece >> 2) * 4 + (lane >> 3);
    if (px >= w || py >= hgt) return;
    const uint32_t i = py * w + px;
    vx_ray r;
    float uv_y;
    camera_ray(cam, px, py, w, hgt, r, &uv_y);
    Hit h;
    cast_ray(s, r.ox, r.oy, r.oz, r.dx, r.dy, r.dz, 0.0f, FLT_MAX_, stkN, stkT, cyc, RENDER_THREADS, h);
    if (hits) store_hit(hits, i, h);
    if (color) store_color(s, color, i, h);
    if (image) {
        // computeLighting (Lighting.glsl:19-28) or the sky gradient
        // (VoxelRayMarch.comp:493-499), stored as RGBA8.
        float cr, cg, cb;
        if (h.flags & F_HIT) {
            float br = 1.0f, bg = 1.0f, bb = 1.0f;
            if (s.color_kind == VX_COLOR_RGBA8) {
                const uint32_t c = __ldg(s.rgba + size_t(h.brick) * 512 + h.voxel);
                br = float(c & 0xFFu) / 255.0f;
                bg = float((c >> 8) & 0xFFu) / 255.0f;
                bb = float((c >> 16) & 0xFFu) / 255.0f;
            } else if (s.color_kind == VX_COLOR_DXT1) {
                dxt_texel(s.dxt, h.brick, h.voxel, br, bg, bb);
            } else if (s.color_kind == VX_COLOR_MATERIAL) {
                // getMaterialColor(voxelData & 0xFF) (VoxelRayMarch.comp:188-192)
                const Rgb m = material_color_shader(__ldg(s.rgba + size_t(h.brick) * 512 + h.voxel) & 0xFFu);
                br = m.r; bg = m.g; bb = m.b;
            }
            const float Ld = (1.0f * 1.0f + 1.0f * 1.0f) + (-1.0f) * (-1.0f);
            const float Linv = 1.0f / sqrtf(Ld);
            const float L[3] = {1.0f * Linv, 1.0f * Linv, -1.0f * Linv};
            float nrm[3] = {0.0f, 0.0f, 0.0f};
            const int axis = (h.flags >> 1) & 3;
            nrm[axis] = (h.flags & F_NEG) ? -1.0f : 1.0f;
            if (s.nrm) {
                // Compressed shading (VoxelRayMarch_Compressed.comp:242-256): the
                // decoded normal blended with the entry-face normal,
                // normalize(n_dxt + face * 0.5).
                float dx, dy, dz;
                dxt_normal(s, h.brick, h.voxel, dx, dy, dz);
                const dxtn::F3 b = dxtn::unit(dxtn::F3{dx, dy, dz} + dxtn::F3{nrm[0], nrm[1], nrm[2]} * 0.5f);
                nrm[0] = b.x; nrm[1] = b.y; nrm[2] = b.z;
            }
            const float nd = (nrm[0] * L[0] + nrm[1] * L[1]) + nrm[2] * L[2];
            const float diffuse = gmax(nd, 0.0f) * 0.7f;
            const float k = 0.3f + diffuse;
            cr = br * k; cg = bg * k; cb = bb * k;
        } else {
            const float k = 1.0f - uv_y * 0.5f;
            cr = 0.5f * k; cg = 0.7f * k; cb = 1.0f * k;
        }
        auto u8 = [](float v) -> uint32_t { return uint32_t(fclamp(v, 0.0f, 1.0f) * 255.0f + 0.5f); };
        image[i] = u8(cr) | (u8(cg) << 8) | (u8(cb) << 16) | (255u << 24);
    }
}

__global__ void camera_rays_kernel(CameraDev cam, uint32_t w, uint32_t hgt, vx_ray* __restrict__ rays) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w * hgt) return;
    vx_ray r;
    camera_ray(cam, i % w, i / w, w, hgt, r, nullptr);
    rays[i] = r;
}

size_t stack_bytes(const DevScene& s, int threads) {
    return (size_t(2) * size_t(s.max_levels) + CYC_WORDS) * size_t(threads) * sizeof(uint32_t);
}

// Stacks of scenes deeper than 15 levels take more than the 48 KiB of dynamic
// shared memory a launch gets without opting in (64 KiB at 23 levels).
template <class K>
cudaError_t allow_smem(K kernel, size_t bytes) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
}

}  // namespace

int launch_cast(const DevScene& s, const vx_ray* rays, uint32_t n, float tmin, float tmax, vx_hit* hits,
                void* color, vx_ray_counters* counters, void* stream, const vx_lod_params* lod) {
    if (n == 0) return int(cudaSuccess);
    const uint32_t grid = (n + BLOCK - 1) / BLOCK;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t smem = stack_bytes(s, BLOCK);
    if (lod && lod->ray_dir_size > 0.0f) {
        if (cudaError_t e = allow_smem(cast_kernel<true>, smem)) return int(e);
        cast_kernel<true><<<grid, BLOCK, smem, st>>>(s, rays, n, tmin, tmax, hits, color, counters,
                                                     LodCone{lod->ray_orig_size, lod->ray_dir_size});
    } else {
        if (cudaError_t e = allow_smem(cast_kernel<false>, smem)) return int(e);
        cast_kernel<false><<<grid, BLOCK, smem, st>>>(s, rays, n, tmin, tmax, hits, color, counters,
                                                      LodCone{0.0f, 0.0f});
    }
    return int(cudaGetLastError());
}

int launch_cast_mapped(const DevScene& s, const vx_ray* rays, uint32_t n_max, const uint32_t* count,
                       const uint32_t* map, float tmin, float tmax, vx_hit* hits, void* stream) {
    if (n_max == 0) return int(cudaSuccess);
    const size_t smem = stack_bytes(s, BLOCK);
    if (cudaError_t e = allow_smem(cast_mapped_kernel, smem)) return int(e);
    cast_mapped_kernel<<<(n_max + BLOCK - 1) / BLOCK, BLOCK, smem, static_cast<cudaStream_t>(stream)>>>(
        s, rays, n_max, count, map, tmin, tmax, hits);
    return int(cudaGetLastError());
}

int launch_render(const DevScene& s, const CameraDev& cam, uint32_t w, uint32_t h, uint32_t* image, vx_hit* hits,
                  void* color, void* stream) {
    const uint64_t n = uint64_t(w) * h;
    if (n == 0) return int(cudaSuccess);
    static_assert(8 % RENDER_WARPS == 0, "a block covers whole 8 x 4 pieces of one 32 x 8 tile");
    const uint64_t grid = uint64_t((w + 31) / 32) * ((h + 7) / 8) * (8 / RENDER_WARPS);
    if (grid > 0x7FFFFFFFull) return int(cudaErrorInvalidValue);
    const size_t smem = stack_bytes(s, RENDER_THREADS);
    if (cudaError_t e = allow_smem(render_kernel, smem)) return int(e);
    render_kernel<<<uint32_t(grid), RENDER_THREADS, smem, static_cast<cudaStream_t>(stream)>>>(s, cam, w, h, image, hits,
                                                                                        color);
    return int(cudaGetLastError());
}

int launch_camera_rays(const CameraDev& cam, uint32_t w, uint32_t h, vx_ray* rays, void* stream) {
    const uint64_t n = uint64_t(w) * h;
    if (n == 0) return int(cudaSuccess);
    camera_rays_kernel<<<uint32_t((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(cam, w, h, rays);
    return int(cudaGetLastError());
}

}  // namespace vx

namespace vx {
VX_VIOLATION_READER(violations_kernels)
}  // namespace vx
