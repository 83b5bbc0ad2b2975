// vx_diff.cu - differentiable form: a forward render that records each
// pixel's hit, and the adjoint kernel that scatters dL/d(colour) into the
// brick attribute pool.  No reference counterpart.
//
// The traversal is discrete and is not differentiated: the forward pass
// records (hit flags, brick, voxel) per pixel and the backward pass replays
// those indices.  Pixel colour of a hit = c * k with the Lambert factor
// k = 0.3 + max(n . L, 0) * 0.7 of shaders/Lighting.glsl:19-28 (L =
// normalize(1,1,-1), n the entry-face normal); a miss shows the sky colour,
// which does not depend on the attributes.
//   kind 0 (per-voxel colour): c = attr[(brick*512 + voxel)*3 + ch]
//   kind 1 (DXT1 endpoints held in FP32 before quantisation): the voxel's
//     block b = brick*32 + (voxel >> 4) has endpoints e0 = attr[b*6 + 0..2],
//     e1 = attr[b*6 + 3..5] and the fixed 2-bit selector s of texel
//     (voxel & 15) in idx[b]; c = w0*e0 + w1*e1 with (w0, w1) = (1, 0),
//     (0, 1), (2/3, 1/3), (1/3, 2/3) for s = 0..3, the interpolation of
//     DXT1ColorCompressor::decodeColorHead (DXT1Compressor.cpp:34-35).
// Loss = sum over pixels and channels of (pixel - target)^2; the adjoint of a
// hit pixel is g = 2 (pixel - target) k, added to dL/dc (kind 0) or w0 g,
// w1 g to dL/de0, dL/de1 (kind 1).  Lanes of a warp that hit the same voxel /
// block are combined first (__match_any_sync + shuffles) so each distinct
// target costs one atomicAdd per channel per warp.

#include "vx_cast.cuh"

namespace vx {
namespace {

constexpr int DBLOCK = 256;
#ifndef VX_DIFF_TILED
#define VX_DIFF_TILED 1
#endif

__device__ __forceinline__ float lambert_k(uint32_t flags) {
    const float Ld = (1.0f * 1.0f + 1.0f * 1.0f) + (-1.0f) * (-1.0f);
    const float Linv = 1.0f / sqrtf(Ld);
    const float L[3] = {1.0f * Linv, 1.0f * Linv, -1.0f * Linv};
    float nrm[3] = {0.0f, 0.0f, 0.0f};
    const int axis = (flags >> 1) & 3;
    nrm[axis] = (flags & F_NEG) ? -1.0f : 1.0f;
    const float nd = (nrm[0] * L[0] + nrm[1] * L[1]) + nrm[2] * L[2];
    return 0.3f + gmax(nd, 0.0f) * 0.7f;
}

__device__ __forceinline__ void dxt_weights(uint32_t sel, float& w0, float& w1) {
    w0 = (sel == 0) ? 1.0f : (sel == 1) ? 0.0f : (sel == 2) ? (2.0f / 3.0f) : (1.0f / 3.0f);
    w1 = (sel == 0) ? 0.0f : (sel == 1) ? 1.0f : (sel == 2) ? (1.0f / 3.0f) : (2.0f / 3.0f);
}

// The cameras of one launch: VX_DIFF_MAX_VIEWS views at most, passed by value
// (kernel parameter space), so a multi-view launch needs no device copy.
struct Views {
    CameraDev cam[VX_DIFF_MAX_VIEWS];
};

// One pixel of the forward pass: cast, record, shade.
__device__ __forceinline__ void forward_pixel(const DevScene& s, const CameraDev& cam, uint32_t px, uint32_t py,
                                              uint32_t w, uint32_t hgt, uint32_t i, int kind,
                                              const float* __restrict__ attr, const uint32_t* __restrict__ idx,
                                              float* __restrict__ image, vx_hit* __restrict__ record,
                                              uint32_t* stkN, float* stkT, uint32_t* cyc, uint32_t stride) {
    vx_ray r;
    float uv_y;
    camera_ray(cam, px, py, w, hgt, r, &uv_y);
    Hit h;
    cast_ray(s, r.ox, r.oy, r.oz, r.dx, r.dy, r.dz, 0.0f, FLT_MAX_, stkN, stkT, cyc, stride, h);
    store_hit(record, i, h);
    float c[3];
    if (h.flags & F_HIT) {
        const float k = lambert_k(h.flags);
        if (kind == 0) {
            const float* a = attr + (size_t(h.brick) * 512 + h.voxel) * 3;
            c[0] = __ldg(a) * k; c[1] = __ldg(a + 1) * k; c[2] = __ldg(a + 2) * k;
        } else {
            const size_t b = size_t(h.brick) * 32 + (h.voxel >> 4);
            const uint32_t sel = (__ldg(idx + b) >> ((h.voxel & 15u) * 2u)) & 3u;
            float w0, w1;
            dxt_weights(sel, w0, w1);
            const float* e = attr + b * 6;
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) c[ch] = (w0 * __ldg(e + ch) + w1 * __ldg(e + 3 + ch)) * k;
        }
    } else {
        const float k = 1.0f - uv_y * 0.5f;
        c[0] = 0.5f * k; c[1] = 0.7f * k; c[2] = 1.0f * k;
    }
    float* o = image + size_t(i) * 3;
    o[0] = c[0]; o[1] = c[1]; o[2] = c[2];
}

// Images and records are view-major: pixel p of view v is entry v * w * hgt + p.
// With VX_DIFF_TILED the work is split into warp tasks of 8 x 4 pixels (the
// eight pieces of a 32 x 8 tile are consecutive tasks), so a warp's rays are
// neighbours in both image directions.  A block holds FWD_WARPS warps, one task
// each: small blocks free their slot as soon as their warps finish, where one
// block per 32 x 8 tile would hold its slot until the slowest of its eight
// warps finished (the orbit views mix rays that hit near with rays that miss far).
#ifndef VX_DIFF_FWD_WARPS
#define VX_DIFF_FWD_WARPS 2
#endif
constexpr int FWD_WARPS = VX_DIFF_FWD_WARPS;
constexpr int FWD_THREADS = VX_DIFF_TILED ? FWD_WARPS * 32 : DBLOCK;

__global__ void __launch_bounds__(FWD_THREADS, 768 / FWD_THREADS) diff_forward_kernel(
    DevScene s, Views views, uint32_t nviews, uint32_t w, uint32_t hgt, int kind, const float* __restrict__ attr,
    const uint32_t* __restrict__ idx, float* __restrict__ image, vx_hit* __restrict__ record) {
    extern __shared__ uint32_t smem[];
    uint32_t* stkN = smem + threadIdx.x;
    float* stkT = reinterpret_cast<float*>(smem + s.max_levels * FWD_THREADS) + threadIdx.x;
    uint32_t* cyc = smem + 2 * s.max_levels * FWD_THREADS + threadIdx.x;
    const uint32_t per_view = w * hgt;
#if VX_DIFF_TILED
    const uint32_t tw = (w + 31) / 32, tiles = tw * ((hgt + 7) / 8);
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t t = uint64_t(blockIdx.x) * FWD_WARPS + (threadIdx.x >> 5);
    if (t >= uint64_t(nviews) * tiles * 8) return;
    const uint32_t piece = uint32_t(t & 7u), tt = uint32_t(t >> 3);
    const uint32_t v = tt / tiles, tl = tt - v * tiles;
    const uint32_t px = (tl % tw) * 32 + (piece & 3u) * 8 + (lane & 7u);
    const uint32_t py = (tl / tw) * 8 + (piece >> 2) * 4 + (lane >> 3);
    if (px >= w || py >= hgt) return;
    forward_pixel(s, views.cam[v], px, py, w, hgt, v * per_view + py * w + px, kind, attr, idx, image, record, stkN,
                  stkT, cyc, FWD_THREADS);
#else
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nviews * per_view) return;
    const uint32_t v = i / per_view, p = i - v * per_view;
    forward_pixel(s, views.cam[v], p % w, p / w, w, hgt, i, kind, attr, idx, image, record, stkN, stkT, cyc, FWD_THREADS);
#endif
}

// Sum v over the lanes of `group` (lanes sharing one key); every lane of the
// group gets the sum.  All lanes of the group call it together.
__device__ __forceinline__ float group_sum(unsigned group, float v) {
    float acc = 0.0f;
    unsigned m = group;
    while (m) {
        const int src = __ffs(m) - 1;
        acc += __shfl_sync(group, v, src);
        m &= m - 1;
    }
    return acc;
}

__global__ void __launch_bounds__(DBLOCK) diff_backward_kernel(uint32_t n, int kind, const uint32_t* __restrict__ idx,
                                                               const vx_hit* __restrict__ record,
                                                               const float* __restrict__ image,
                                                               const float* __restrict__ target,
                                                               float* __restrict__ grad, float* __restrict__ loss) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = i < n;
    uint4 rec = make_uint4(0, 0xFFFFFFFFu, 0, 0);
    float d[3] = {0.0f, 0.0f, 0.0f};
    if (in) {
        rec = reinterpret_cast<const uint4*>(record)[i];
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) d[ch] = image[size_t(i) * 3 + ch] - target[size_t(i) * 3 + ch];
    }
    // loss: block reduction, one atomicAdd per block
    if (loss) {
        float l = (d[0] * d[0] + d[1] * d[1]) + d[2] * d[2];
        for (int off = 16; off > 0; off >>= 1) l += __shfl_down_sync(0xFFFFFFFFu, l, off);
        __shared__ float part[DBLOCK / 32];
        if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = l;
        __syncthreads();
        if (threadIdx.x < 32) {
            float v = threadIdx.x < DBLOCK / 32 ? part[threadIdx.x] : 0.0f;
            for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, off);
            if (threadIdx.x == 0) atomicAdd(loss, v);
        }
    }
    const uint32_t flags = (rec.w >> 16) & 0xFFu;
    const bool hit = in && (flags & F_HIT);
    const uint32_t brick = rec.y, voxel = rec.w & 0xFFFFu;
    float g[3] = {0.0f, 0.0f, 0.0f};
    unsigned long long key = ~0ull;
    float w0 = 0.0f, w1 = 0.0f;
    if (hit) {
        const float k = lambert_k(flags);
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) g[ch] = 2.0f * d[ch] * k;
        if (kind == 0) {
            key = uint64_t(brick) * 512 + voxel;
        } else {
            key = uint64_t(brick) * 32 + (voxel >> 4);
            const uint32_t sel = (__ldg(idx + key) >> ((voxel & 15u) * 2u)) & 3u;
            dxt_weights(sel, w0, w1);
        }
    }
    const unsigned group = __match_any_sync(0xFFFFFFFFu, key);
    if (key == ~0ull) return;
    const bool leader = (__ffs(group) - 1) == int(threadIdx.x & 31);
    if (kind == 0) {
        float s3[3];
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) s3[ch] = group_sum(group, g[ch]);
        if (leader) {
            float* dst = grad + key * 3;
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) atomicAdd(dst + ch, s3[ch]);
        }
    } else {
        float s6[6];
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) {
            s6[ch] = group_sum(group, w0 * g[ch]);
            s6[3 + ch] = group_sum(group, w1 * g[ch]);
        }
        if (leader) {
            float* dst = grad + key * 6;
#pragma unroll
            for (int j = 0; j < 6; ++j) atomicAdd(dst + j, s6[j]);
        }
    }
}

}  // namespace
}  // namespace vx

extern "C" int vx_diff_forward_views(const vx_scene* scene, const vx_camera_pc* pcs, uint32_t views, uint32_t w,
                                     uint32_t h, int32_t kind, const float* attr, const uint32_t* dxt_idx,
                                     float* image, vx_hit* record, void* stream) {
    using namespace vx;
    if (!scene || !pcs || !attr || !image || !record || (kind == 1 && !dxt_idx) || (kind != 0 && kind != 1))
        return fail(VX_EINVAL, "vx_diff_forward: bad argument");
    if (views > VX_DIFF_MAX_VIEWS)
        return fail(VX_EOVERFLOW, "vx_diff_forward_views: more than VX_DIFF_MAX_VIEWS views in one call");
    const uint64_t n = uint64_t(w) * h * views;
    if (n > 0xFFFFFFFFull) return fail(VX_EOVERFLOW, "vx_diff_forward: views * width * height exceeds 2^32");
    if (reinterpret_cast<uintptr_t>(record) % 16 || reinterpret_cast<uintptr_t>(image) % 4)
        return fail(VX_EINVAL, "vx_diff_forward: misaligned output");
    if (n == 0) return VX_OK;
    const DevScene& s = scene_dev(scene);
    Views v{};
    for (uint32_t k = 0; k < views; ++k) v.cam[k] = camera_from_pc(pcs[k]);
    const size_t smem = (size_t(2) * size_t(s.max_levels) + CYC_WORDS) * FWD_THREADS * sizeof(uint32_t);
    // stacks of scenes deeper than 15 levels need more than 48 KiB per 256 threads
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(diff_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   int(smem));
        if (e != cudaSuccess) return fail(VX_ECUDA, std::string("vx_diff_forward: ") + cudaGetErrorString(e));
    }
#if VX_DIFF_TILED
    const uint64_t tasks = uint64_t(views) * ((w + 31) / 32) * ((h + 7) / 8) * 8;
    const uint64_t blocks = (tasks + FWD_WARPS - 1) / FWD_WARPS;
#else
    const uint64_t blocks = (n + DBLOCK - 1) / DBLOCK;
#endif
    if (blocks > 0x7FFFFFFFull) return fail(VX_EOVERFLOW, "vx_diff_forward: too many pixels for one launch");
    diff_forward_kernel<<<uint32_t(blocks), FWD_THREADS, smem, static_cast<cudaStream_t>(stream)>>>(
        s, v, views, w, h, kind, attr, dxt_idx, image, record);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VX_OK : fail(VX_ECUDA, std::string("vx_diff_forward: ") + cudaGetErrorString(e));
}

extern "C" int vx_diff_forward(const vx_scene* scene, const vx_camera_pc* pc, uint32_t w, uint32_t h, int32_t kind,
                               const float* attr, const uint32_t* dxt_idx, float* image, vx_hit* record,
                               void* stream) {
    if (!pc) return vx::fail(VX_EINVAL, "vx_diff_forward: bad argument");
    return vx_diff_forward_views(scene, pc, 1, w, h, kind, attr, dxt_idx, image, record, stream);
}

extern "C" int vx_diff_backward(uint32_t n, int32_t kind, const uint32_t* dxt_idx, const vx_hit* record,
                                const float* image, const float* target, float* grad, float* loss, void* stream) {
    using namespace vx;
    if ((n && (!record || !image || !target || !grad)) || (kind == 1 && !dxt_idx) || (kind != 0 && kind != 1))
        return fail(VX_EINVAL, "vx_diff_backward: bad argument");
    if (n == 0) return VX_OK;
    diff_backward_kernel<<<(n + DBLOCK - 1) / DBLOCK, DBLOCK, 0, static_cast<cudaStream_t>(stream)>>>(
        n, kind, dxt_idx, record, image, target, grad, loss);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VX_OK : fail(VX_ECUDA, std::string("vx_diff_backward: ") + cudaGetErrorString(e));
}

namespace vx {
VX_VIOLATION_READER(violations_diff)
}  // namespace vx
