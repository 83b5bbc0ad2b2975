// vx_synth.cu - the value-noise occupancy generator on the device.
//
// Produces exactly the bits of vx_synth_noise (vx_build.cpp): the same lattice
// hash, the same binary32 operation order per voxel (the kernels are built
// with --fmad=false), and the same threshold, the value of ascending rank
// N - round(fill * N), found here by a three-pass radix select over the
// values' bit patterns (12 + 12 + 8 bits) with shared-memory histograms.
#include <cstdint>
#include <vector>

#include "vx_hash.h"
#include "vx_internal.h"

namespace vx {
namespace {

struct OctDev {
    uint32_t s, cells;
    float amp;
    const float* lat;
};
struct NoiseParams {
    uint32_t R, octaves;
    OctDev oct[16];
};

__global__ void lattice_kernel(float* lat, uint32_t c, uint32_t o, uint64_t seed) {
    const uint64_t n = uint64_t(c) * c * c;
    for (uint64_t t = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; t < n; t += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t i = uint32_t(t % c), j = uint32_t((t / c) % c), k = uint32_t(t / (uint64_t(c) * c));
        lat[t] = float(hash4(seed, o, i, j, k) >> 40) * (1.0f / 16777216.0f);
    }
}

// One thread per voxel, x fastest; same expression order as the host row loop.
__global__ void field_kernel(NoiseParams p, float* field) {
    const uint64_t R = p.R, N = R * R * R;
    for (uint64_t t = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; t < N; t += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t x = uint32_t(t % R), y = uint32_t((t / R) % R), z = uint32_t(t / (R * R));
        float out = 0.0f;
        for (uint32_t o = 0; o < p.octaves; ++o) {
            const OctDev q = p.oct[o];
            const float fs = float(q.s);
            const float py = (float(y) + 0.5f) / fs, pz = (float(z) + 0.5f) / fs;
            const float jy = floorf(py), kz = floorf(pz);
            const float fy = py - jy, fz = pz - kz;
            const float wy = fy * fy * (3.0f - 2.0f * fy), wz = fz * fz * (3.0f - 2.0f * fz);
            const uint32_t j = uint32_t(jy), k = uint32_t(kz);
            const float px = (float(x) + 0.5f) / fs;
            const float ix = floorf(px);
            const float fx = px - ix;
            const float wx = fx * fx * (3.0f - 2.0f * fx);
            const uint32_t i = uint32_t(ix);
            const uint32_t c = q.cells;
            float lz[2];
#pragma unroll
            for (int di = 0; di < 2; ++di) {
                const uint32_t ii = i + di;
                const float a0 = __ldg(q.lat + (size_t(k) * c + j) * c + ii);
                const float b0 = __ldg(q.lat + (size_t(k) * c + j + 1) * c + ii);
                const float a1 = __ldg(q.lat + (size_t(k + 1) * c + j) * c + ii);
                const float b1 = __ldg(q.lat + (size_t(k + 1) * c + j + 1) * c + ii);
                const float ly0 = a0 + wy * (b0 - a0);
                const float ly1 = a1 + wy * (b1 - a1);
                lz[di] = ly0 + wz * (ly1 - ly0);
            }
            const float v = lz[0] + wx * (lz[1] - lz[0]);
            out = out + q.amp * v;
        }
        field[t] = out;
    }
}

// Histogram of (bits >> shift) & (nbins - 1) over values whose bits match
// prefix under prefix_mask.
__global__ void histo_kernel(const uint32_t* __restrict__ vals, uint64_t n, uint32_t prefix_mask, uint32_t prefix,
                             int shift, uint32_t nbins, unsigned long long* __restrict__ out) {
    __shared__ uint32_t h[4096];
    for (uint32_t b = threadIdx.x; b < nbins; b += blockDim.x) h[b] = 0;
    __syncthreads();
    for (uint64_t t = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; t < n; t += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t u = __ldg(vals + t);
        if ((u & prefix_mask) == prefix) atomicAdd(&h[(u >> shift) & (nbins - 1)], 1u);
    }
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < nbins; b += blockDim.x)
        if (h[b]) atomicAdd(out + b, (unsigned long long)h[b]);
}

__global__ void pack_kernel(const float* __restrict__ field, uint32_t R, uint32_t thr_bits, int any_solid, int shell,
                            uint64_t* __restrict__ bits) {
    const uint64_t wpr = R / 64, W = uint64_t(R) * R * wpr;
    const float thr = __uint_as_float(thr_bits);
    for (uint64_t w = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; w < W; w += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t row = w / wpr;
        const uint32_t y = uint32_t(row % R), z = uint32_t(row / R);
        const uint32_t x0 = uint32_t(w % wpr) * 64;
        uint64_t word = 0;
        for (uint32_t b = 0; b < 64; ++b) {
            const uint32_t x = x0 + b;
            bool solid = any_solid && field[row * R + x] >= thr;
            if (shell && (x == 0 || y == 0 || z == 0 || x == R - 1 || y == R - 1 || z == R - 1)) solid = true;
            word |= uint64_t(solid) << b;
        }
        bits[w] = word;
    }
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
};

}  // namespace
}  // namespace vx

static int vx_synth_noise_dev_body(uint32_t R, uint32_t spacing, uint32_t octaves, float fill, uint64_t seed,
                                  int32_t shell, uint64_t* out_bits_dev, void* stream) {
    using namespace vx;
    if (!out_bits_dev || R < 64 || R % 64 != 0 || R > 2048 || octaves < 1 || octaves > 16 || spacing < 1 ||
        (spacing >> (octaves - 1)) < 1 || !(fill >= 0.0f && fill <= 1.0f))
        return fail(VX_EINVAL, "vx_synth_noise_dev: bad arguments");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint64_t N = uint64_t(R) * R * R;
    NoiseParams p{};
    p.R = R;
    p.octaves = octaves;
    std::vector<DevBuf> lat(octaves);
    float amp = 1.0f;
    auto cerr = [](cudaError_t e, const char* w) {
        return fail(VX_ECUDA, std::string("vx_synth_noise_dev: ") + w + ": " + cudaGetErrorString(e));
    };
    for (uint32_t o = 0; o < octaves; ++o) {
        OctDev& q = p.oct[o];
        q.s = spacing >> o;
        q.amp = amp;
        amp *= 0.5f;
        q.cells = (R + q.s - 1) / q.s + 2;
        const uint64_t n = uint64_t(q.cells) * q.cells * q.cells;
        cudaError_t e = cudaMalloc(&lat[o].p, n * 4);
        if (e != cudaSuccess) return cerr(e, "cudaMalloc");
        lattice_kernel<<<1184, 256, 0, st>>>(static_cast<float*>(lat[o].p), q.cells, o, seed);
        q.lat = static_cast<const float*>(lat[o].p);
    }
    DevBuf field, hist;
    cudaError_t e = cudaMalloc(&field.p, N * 4);
    if (e != cudaSuccess) return cerr(e, "cudaMalloc field");
    e = cudaMalloc(&hist.p, 4096 * sizeof(unsigned long long));
    if (e != cudaSuccess) return cerr(e, "cudaMalloc histogram");
    field_kernel<<<148 * 16, 256, 0, st>>>(p, static_cast<float*>(field.p));
    e = cudaGetLastError();
    if (e != cudaSuccess) return cerr(e, "field_kernel");
    const uint64_t n_solid = uint64_t(double(fill) * double(N) + 0.5);
    uint32_t thr_bits = 0xFFFFFFFFu;
    if (n_solid > 0) {
        uint64_t r = N - n_solid;
        uint32_t prefix = 0, mask = 0;
        const int shifts[3] = {20, 8, 0};
        const uint32_t nb[3] = {4096, 4096, 256};
        std::vector<unsigned long long> h(4096);
        for (int pass = 0; pass < 3; ++pass) {
            cudaMemsetAsync(hist.p, 0, 4096 * sizeof(unsigned long long), st);
            histo_kernel<<<148 * 8, 512, 0, st>>>(static_cast<const uint32_t*>(field.p), N, mask, prefix,
                                                  shifts[pass], nb[pass],
                                                  static_cast<unsigned long long*>(hist.p));
            e = cudaMemcpyAsync(h.data(), hist.p, nb[pass] * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return cerr(e, "histogram");
            uint64_t acc = 0;
            uint32_t bin = nb[pass] - 1;
            for (uint32_t b = 0; b < nb[pass]; ++b) {
                if (acc + h[b] > r) { bin = b; break; }
                acc += h[b];
            }
            r -= acc;
            prefix |= bin << shifts[pass];
            mask |= (nb[pass] - 1) << shifts[pass];
        }
        thr_bits = prefix;
    }
    pack_kernel<<<148 * 8, 256, 0, st>>>(static_cast<const float*>(field.p), R, thr_bits, n_solid > 0 ? 1 : 0, shell,
                                         out_bits_dev);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cerr(e, "pack_kernel");
    return VX_OK;
}

extern "C" int vx_synth_noise_dev(uint32_t R, uint32_t spacing, uint32_t octaves, float fill, uint64_t seed,
                                  int32_t shell, uint64_t* out_bits_dev, void* stream) {
    return vx::guarded("vx_synth_noise_dev", [&] { return vx_synth_noise_dev_body(R, spacing, octaves, fill, seed, shell, out_bits_dev, stream); });
}
