// vx_payload.cu - the compressed brick payloads the rebuild writes
// (SVORebuild.cpp:615-722): DXT normal blocks from geometric normals and DXT1
// colour blocks from per-voxel colours, each built on the GPU (one thread per
// 16-voxel block) or on the host from the same code; and the per-hit normal
// decode of the compressed shader (getCompressedVoxelNormal,
// VoxelRayMarch_Compressed.comp:160-165).
#include <algorithm>
#include <thread>
#include <vector>

#include "vx_cast.cuh"
#include "vx_dxt1.h"
#include "vx_dxtn.h"
#include "vx_palette.h"

namespace vx {
namespace {

// MaterialIdToColor of every material word (grid-stride).
__global__ void material_rgb_kernel(const uint32_t* __restrict__ words, uint64_t n, float* __restrict__ rgb) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const Rgb c = material_color_payload(words[i]);
        rgb[3 * i] = c.r;
        rgb[3 * i + 1] = c.g;
        rgb[3 * i + 2] = c.b;
    }
}

// Thread i encodes block i & 31 of brick i >> 5.  The 32 threads of a warp
// share one brick, so the occupancy words a thread reads (at most 6 of the
// brick's 16) come from the same 64 bytes in L1; each thread writes its
// 16-byte block, a warp 512 contiguous bytes.  The 27 neighbour-code normals
// sit in shared memory, one 16-byte entry each.
__global__ void __launch_bounds__(128) build_normals_kernel(const uint32_t* __restrict__ occ, uint64_t blocks,
                                                            uint4* __restrict__ out) {
    __shared__ float4 tab[dxtn::NUM_CODES];
    if (threadIdx.x < dxtn::NUM_CODES) tab[threadIdx.x] = dxtn::code_entry(int(threadIdx.x));
    __syncthreads();
    const dxtn::CodeTable lookup{tab};
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < blocks;
         i += uint64_t(gridDim.x) * blockDim.x) {
        uint64_t a, b;
        dxtn::brick_block(occ + (i >> 5) * 16, int(i & 31), lookup, a, b);
        out[i] = make_uint4(uint32_t(a), uint32_t(a >> 32), uint32_t(b), uint32_t(b >> 32));
    }
}

// One warp per brick: the brick's 512 RGB texels (6 KiB) come in with
// coalesced loads (16-byte loads when the colours are 16-byte aligned) and are
// staged in shared memory with a 49-word stride per 16-texel block, so that the
// lanes' texel reads (lane k = block k) fall in 32 different banks; lane k then
// encodes block k and the warp writes its 256 output bytes contiguously.
constexpr int DXT1_WARPS = 4;
constexpr int DXT1_STRIDE = 49;

template <bool VEC>
__global__ void __launch_bounds__(DXT1_WARPS * 32) build_dxt1_kernel(const float* __restrict__ rgb,
                                                                     const uint32_t* __restrict__ occ,
                                                                     uint64_t bricks, uint64_t* __restrict__ out) {
    __shared__ float stage[DXT1_WARPS][32 * DXT1_STRIDE];
    const int lane = threadIdx.x & 31;
    float* s = stage[threadIdx.x >> 5];
    for (uint64_t brick = uint64_t(blockIdx.x) * DXT1_WARPS + (threadIdx.x >> 5); brick < bricks;
         brick += uint64_t(gridDim.x) * DXT1_WARPS) {
        const float* src = rgb + brick * 1536;
        if (VEC) {
            for (int q = lane; q < 384; q += 32) {  // 12 float4 per block
                const float4 v = __ldg(reinterpret_cast<const float4*>(src) + q);
                float* d = s + (q / 12) * DXT1_STRIDE + (q % 12) * 4;
                d[0] = v.x;
                d[1] = v.y;
                d[2] = v.z;
                d[3] = v.w;
            }
        } else {
            for (int f = lane; f < 1536; f += 32) s[(f / 48) * DXT1_STRIDE + f % 48] = __ldg(src + f);
        }
        __syncwarp();
        const uint32_t o = (__ldg(occ + brick * 16 + (lane >> 1)) >> ((lane & 1) * 16)) & 0xFFFFu;
        float* mine = s + lane * DXT1_STRIDE;
        uint64_t block = 0;
        if (o) {
            dxt1::mask_empty(mine, o);
            block = dxt1::encode16(mine);
        }
        out[brick * 32 + lane] = block;
        __syncwarp();
    }
}

// normalize(decode) of each hit voxel's texel; zeros on a miss or an LOD hit.
__global__ void __launch_bounds__(256) hit_normals_kernel(DevScene s, const uint4* __restrict__ hits, uint32_t n,
                                                          float* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint4 h = __ldg(hits + i);
    float x = 0.0f, y = 0.0f, z = 0.0f;
    const uint32_t flags = (h.w >> 16) & 0xFFu;
    if ((flags & F_HIT) && h.y != NONE) dxt_normal(s, h.y, h.w & 0xFFFFu, x, y, z);
    out[size_t(i) * 3] = x;
    out[size_t(i) * 3 + 1] = y;
    out[size_t(i) * 3 + 2] = z;
}

int cuda_err(cudaError_t e, const char* what) {
    return fail(VX_ECUDA, std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

}  // namespace
}  // namespace vx

extern "C" int vx_build_normals_dev(const uint32_t* occ_dev, uint32_t brick_count, uint64_t* out_dev, void* stream) {
    using namespace vx;
    if (brick_count && (!occ_dev || !out_dev)) return fail(VX_EINVAL, "vx_build_normals_dev: null argument");
    if (reinterpret_cast<uintptr_t>(occ_dev) % 16 || reinterpret_cast<uintptr_t>(out_dev) % 16)
        return fail(VX_EINVAL, "vx_build_normals_dev: buffers need 16-byte alignment");
    if (brick_count == 0) return VX_OK;
    const uint64_t blocks = uint64_t(brick_count) * 32;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t want = (blocks + 127) / 128;
    const uint32_t grid = uint32_t(std::min<uint64_t>(want, uint64_t(sms) * 64));
    build_normals_kernel<<<grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(occ_dev, blocks,
                                                                             reinterpret_cast<uint4*>(out_dev));
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VX_OK : cuda_err(e, "vx_build_normals_dev");
}

static int vx_build_normals_body(const uint32_t* occ, uint32_t brick_count, uint64_t* out) {
    using namespace vx;
    if (brick_count && (!occ || !out)) return fail(VX_EINVAL, "vx_build_normals: null argument");
    const unsigned T = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    float4 tab[dxtn::NUM_CODES];
    for (int c = 0; c < dxtn::NUM_CODES; ++c) tab[c] = dxtn::code_entry(c);
    const dxtn::CodeTable lookup{tab};
    auto work = [&](uint64_t b0, uint64_t b1) {
        for (uint64_t b = b0; b < b1; ++b)
            for (int k = 0; k < 32; ++k)
                dxtn::brick_block(occ + 16 * b, k, lookup, out[(b * 32 + k) * 2], out[(b * 32 + k) * 2 + 1]);
    };
    if (T == 1 || brick_count < 256) {
        work(0, brick_count);
        return VX_OK;
    }
    std::vector<std::thread> th;
    const uint64_t chunk = (uint64_t(brick_count) + T - 1) / T;
    for (unsigned t = 0; t < T; ++t) {
        const uint64_t b0 = uint64_t(t) * chunk, b1 = std::min<uint64_t>(brick_count, b0 + chunk);
        if (b0 >= b1) break;
        th.emplace_back(work, b0, b1);
    }
    for (auto& x : th) x.join();
    return VX_OK;
}

extern "C" int vx_build_normals(const uint32_t* occ, uint32_t brick_count, uint64_t* out) {
    return vx::guarded("vx_build_normals", [&] { return vx_build_normals_body(occ, brick_count, out); });
}

extern "C" int vx_build_dxt1_dev(const float* rgb_dev, const uint32_t* occ_dev, uint32_t brick_count,
                                 uint64_t* out_dev, void* stream) {
    using namespace vx;
    if (brick_count && (!rgb_dev || !occ_dev || !out_dev)) return fail(VX_EINVAL, "vx_build_dxt1_dev: null argument");
    if (reinterpret_cast<uintptr_t>(occ_dev) % 16 || reinterpret_cast<uintptr_t>(out_dev) % 8 ||
        reinterpret_cast<uintptr_t>(rgb_dev) % 4)
        return fail(VX_EINVAL, "vx_build_dxt1_dev: misaligned buffer");
    if (brick_count == 0) return VX_OK;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint32_t grid =
        uint32_t(std::min<uint64_t>((uint64_t(brick_count) + DXT1_WARPS - 1) / DXT1_WARPS, uint64_t(sms) * 32));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (reinterpret_cast<uintptr_t>(rgb_dev) % 16 == 0)
        build_dxt1_kernel<true><<<grid, DXT1_WARPS * 32, 0, st>>>(rgb_dev, occ_dev, brick_count, out_dev);
    else
        build_dxt1_kernel<false><<<grid, DXT1_WARPS * 32, 0, st>>>(rgb_dev, occ_dev, brick_count, out_dev);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VX_OK : cuda_err(e, "vx_build_dxt1_dev");
}

static int vx_build_dxt1_body(const float* rgb, const uint32_t* occ, uint32_t brick_count, uint64_t* out) {
    using namespace vx;
    if (brick_count && (!rgb || !occ || !out)) return fail(VX_EINVAL, "vx_build_dxt1: null argument");
    const unsigned T = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    auto work = [&](uint64_t b0, uint64_t b1) {
        for (uint64_t b = b0; b < b1; ++b)
            for (int k = 0; k < 32; ++k) out[b * 32 + k] = dxt1::brick_block(rgb + b * 512 * 3, occ + 16 * b, k);
    };
    if (T == 1 || brick_count < 256) {
        work(0, brick_count);
        return VX_OK;
    }
    std::vector<std::thread> th;
    const uint64_t chunk = (uint64_t(brick_count) + T - 1) / T;
    for (unsigned t = 0; t < T; ++t) {
        const uint64_t b0 = uint64_t(t) * chunk, b1 = std::min<uint64_t>(brick_count, b0 + chunk);
        if (b0 >= b1) break;
        th.emplace_back(work, b0, b1);
    }
    for (auto& x : th) x.join();
    return VX_OK;
}

extern "C" int vx_build_dxt1(const float* rgb, const uint32_t* occ, uint32_t brick_count, uint64_t* out) {
    return vx::guarded("vx_build_dxt1", [&] { return vx_build_dxt1_body(rgb, occ, brick_count, out); });
}

static int vx_material_rgb_body(const uint32_t* words, uint64_t n, float* rgb) {
    if (n && (!words || !rgb)) return vx::fail(VX_EINVAL, "vx_material_rgb: null argument");
    const unsigned T = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    auto work = [&](uint64_t a, uint64_t b) {
        for (uint64_t i = a; i < b; ++i) {
            const vx::Rgb c = vx::material_color_payload(words[i]);
            rgb[3 * i] = c.r;
            rgb[3 * i + 1] = c.g;
            rgb[3 * i + 2] = c.b;
        }
    };
    if (T == 1 || n < (uint64_t(1) << 16)) {
        work(0, n);
        return VX_OK;
    }
    std::vector<std::thread> th;
    const uint64_t chunk = (n + T - 1) / T;
    for (unsigned t = 0; t < T; ++t) {
        const uint64_t a = uint64_t(t) * chunk, b = std::min(n, a + chunk);
        if (a >= b) break;
        th.emplace_back(work, a, b);
    }
    for (auto& x : th) x.join();
    return VX_OK;
}

extern "C" int vx_material_rgb(const uint32_t* words, uint64_t n, float* rgb) {
    return vx::guarded("vx_material_rgb", [&] { return vx_material_rgb_body(words, n, rgb); });
}

extern "C" int vx_material_rgb_dev(const uint32_t* words, uint64_t n, float* rgb, void* stream) {
    using namespace vx;
    if (n && (!words || !rgb)) return fail(VX_EINVAL, "vx_material_rgb_dev: null argument");
    if (reinterpret_cast<uintptr_t>(words) % 4 || reinterpret_cast<uintptr_t>(rgb) % 4)
        return fail(VX_EINVAL, "vx_material_rgb_dev: misaligned buffer");
    if (n == 0) return VX_OK;
    const uint64_t blocks = std::min<uint64_t>((n + 255) / 256, 148 * 16);
    material_rgb_kernel<<<unsigned(blocks), 256, 0, static_cast<cudaStream_t>(stream)>>>(words, n, rgb);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VX_OK : cuda_err(e, "vx_material_rgb_dev");
}

extern "C" int vx_hit_normals(const vx_scene* scene, const vx_hit* hits_dev, uint32_t n, float* normals_dev,
                              void* stream) {
    using namespace vx;
    if (!scene || (n && (!hits_dev || !normals_dev))) return fail(VX_EINVAL, "vx_hit_normals: null argument");
    const DevScene& s = scene_dev(scene);
    if (!s.nrm) return fail(VX_EINVAL, "vx_hit_normals: the scene has no normal payload");
    if (reinterpret_cast<uintptr_t>(hits_dev) % 16 || reinterpret_cast<uintptr_t>(normals_dev) % 4)
        return fail(VX_EINVAL, "vx_hit_normals: misaligned buffer");
    if (n == 0) return VX_OK;
    hit_normals_kernel<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        s, reinterpret_cast<const uint4*>(hits_dev), n, normals_dev);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VX_OK : cuda_err(e, "vx_hit_normals");
}

namespace vx {
VX_VIOLATION_READER(violations_payload)
}  // namespace vx
