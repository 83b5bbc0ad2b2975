// vx_batch.cu - batched form: rays of many scenes in one persistent launch,
// bounce / shadow ray generation, the frame CUDA graph and the autotuner.
//
// The batched kernel is persistent: one grid of (SM count x resident blocks)
// whose warps take tasks of K consecutive rays from a global work counter
// (atomicAdd by lane 0, broadcast with __shfl_sync).  The rays of all scenes
// sit in one buffer; ray r belongs to the scene i with begin[i] <= r <
// begin[i+1], found by binary search over a copy of begin[] and of the scene
// table in shared memory, so a task may span two scenes.  Each lane walks its
// rays of the task independently (independent thread scheduling lets lanes
// that finish early take their next ray while others are still traversing);
// the warp re-converges at the next task fetch.  The per-ray traversal is the
// one of the plain kernel (vx_cast.cuh), so hits are identical bit for bit.
// Static lanes may take an iteration budget: rays still running after it are
// listed and cast again from the start by a second launch over the list.
// The frame (vx_batch_capture_frame_compact) casts only the bounce rays of
// primary hits, grouped per scene by direction bin; vx_batch_capture_frame_parts
// captures it in parts whose host copies overlap the other parts' casts.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "vx_cast.cuh"

namespace vx {
namespace {

constexpr int MAX_LEVELS_ALL = 23;
constexpr uint32_t NUM_BOUNCE_DIRS = 4096;

// Cosine-weighted hemisphere directions about +z (device copy of bounce_table()).
__device__ float g_bounce_dirs[NUM_BOUNCE_DIRS * 3];

struct BatchArgs {
    const DevScene* scenes;
    uint32_t S;
    const uint32_t* begin;  // S + 1 prefix offsets
    const vx_ray* rays;
    uint32_t n;
    float tmin, tmax;
    vx_hit* hits;
    vx_ray_counters* counters;
    uint32_t* work;  // task counter, zero before the launch
    uint32_t K;      // rays per warp task
    int maxL;        // largest max_levels in the batch
    int refill;      // refill idle lanes once this many are idle (refilling kernels)
    const uint32_t* map = nullptr;    // hit / counter slot of ray r (null: slot r)
    const uint32_t* n_dev = nullptr;  // ray count known on the device only (null: n)
    // Static lanes with an iteration budget: a ray still running after
    // `budget` iterations is appended to retry[0 .. *retry_n) instead of being
    // finished.  A second launch with gather = retry casts exactly those rays
    // (task ray j is ray gather[j]).
    int budget = 0;
    uint32_t* retry = nullptr;
    uint32_t* retry_n = nullptr;
    const uint32_t* gather = nullptr;
};

// Rays of the launch: n, or the device-side count when the rays were
// compacted on the device (at most n).
__device__ __forceinline__ uint32_t ray_count(const BatchArgs& a) {
    return a.n_dev ? min(a.n, __ldg(a.n_dev)) : a.n;
}

__device__ __forceinline__ uint32_t out_slot(const BatchArgs& a, uint32_t r) {
    return a.map ? __ldg(a.map + r) : r;
}

__device__ __forceinline__ int scene_of(const uint32_t* beg, uint32_t S, uint32_t r) {
    int lo = 0, hi = int(S);
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (beg[mid] <= r) lo = mid;
        else hi = mid;
    }
    return int(bounded(uint32_t(lo), S, V_SCENE));
}

__device__ __forceinline__ void store_counters(vx_ray_counters* counters, uint32_t r, const Hit& h) {
    if (!counters) return;
    uint4 rc;
    rc.x = (h.iters & 0xFFFFu) | (h.grid_reads << 16);
    rc.y = h.dda_steps;
    rc.z = (h.run_iters & 0xFFFFu) | (h.run_grid_reads << 16);
    rc.w = h.run_dda_steps;
    reinterpret_cast<uint4*>(counters)[r] = rc;
}

// Refilling variant: a lane keeps its ray's traversal state in registers and
// advances it one ESVO iteration per round; when at least `refill` lanes of
// the warp are idle, the warp deals the next rays of its task to them (rank
// among the idle lanes by __ballot_sync / __popc) and takes a new task from
// the work counter when the current one is used up.  Every warp-wide
// primitive runs with all 32 lanes converged; the traversal between them is
// per lane.
template <int BLOCK, int MINB, bool SMEM_STACK>
__global__ void __launch_bounds__(BLOCK, MINB) batch_refill_kernel(BatchArgs a) {
    extern __shared__ uint32_t smem[];
    DevScene* sc = reinterpret_cast<DevScene*>(smem);
    uint32_t* beg = reinterpret_cast<uint32_t*>(sc + a.S);
    {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(a.scenes);
        uint32_t* dst = reinterpret_cast<uint32_t*>(sc);
        const uint32_t words = a.S * uint32_t(sizeof(DevScene) / 4);
        for (uint32_t i = threadIdx.x; i < words; i += BLOCK) dst[i] = src[i];
        for (uint32_t i = threadIdx.x; i <= a.S; i += BLOCK) beg[i] = a.begin[i];
    }
    __syncthreads();
    uint32_t* stk_base = beg + ((a.S + 1 + 3) & ~3u);
    uint32_t lnode[SMEM_STACK ? 1 : MAX_LEVELS_ALL];
    float ltmax[SMEM_STACK ? 1 : MAX_LEVELS_ALL];
    uint32_t lcyc[SMEM_STACK ? 1 : CYC_WORDS];
    uint32_t* stkN;
    float* stkT;
    uint32_t* cyc;
    int stride;
    if (SMEM_STACK) {
        stkN = stk_base + threadIdx.x;
        stkT = reinterpret_cast<float*>(stk_base + a.maxL * BLOCK) + threadIdx.x;
        cyc = stk_base + 2 * a.maxL * BLOCK + threadIdx.x;
        stride = BLOCK;
    } else {
        stkN = lnode;
        stkT = ltmax;
        cyc = lcyc;
        stride = 1;
    }
    const uint32_t FULL = 0xFFFFFFFFu;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t below = (1u << lane) - 1u;
    const uint32_t n = ray_count(a);
    uint64_t next = 0, end = 0;  // warp-uniform cursor into the current task
    bool tasks_left = true;
    bool active = false;
    uint32_t ray = 0;
    int sid = 0;
    CastState st;
    uint32_t ck[CK_WORDS];
    for (;;) {
        uint32_t idle = __ballot_sync(FULL, !active);
        if (__popc(idle) >= a.refill || idle == FULL) {
            while (idle) {
                if (next >= end) {
                    if (!tasks_left) break;
                    uint32_t t = 0;
                    if (lane == 0) t = atomicAdd(a.work, 1u);
                    t = __shfl_sync(FULL, t, 0);
                    next = uint64_t(t) * a.K;
                    if (next >= n) { tasks_left = false; next = end = 0; break; }
                    end = min(next + a.K, uint64_t(n));
                }
                const uint32_t avail = uint32_t(end - next);
                const uint32_t rank = __popc(idle & below);
                const bool got = ((idle >> lane) & 1u) && rank < avail;
                const uint32_t taken = min(avail, uint32_t(__popc(idle)));
                if (got) {
                    ray = uint32_t(next) + rank;
                    sid = scene_of(beg, a.S, ray);
                    const float2* r2 = reinterpret_cast<const float2*>(a.rays + ray);
                    const float2 p = __ldg(r2), q = __ldg(r2 + 1), w = __ldg(r2 + 2);
                    if (cast_init(sc[sid], p.x, p.y, q.x, q.y, w.x, w.y, a.tmin, a.tmax, stkN, stkT, stride, st)) {
                        store_hit(a.hits, out_slot(a, ray), st.h);
                        store_counters(a.counters, out_slot(a, ray), st.h);
                    } else {
                        active = true;
                    }
                }
                next += taken;
                idle = __ballot_sync(FULL, !active);
            }
        }
        if (__ballot_sync(FULL, active) == 0) {
            if (!tasks_left && next >= end) break;
            continue;
        }
        if (active && cast_step<false, !SMEM_STACK, true>(sc[sid], st, stkN, stkT, cyc, stride, ck)) {
            finish_skipped(st, ck);
            store_hit(a.hits, out_slot(a, ray), st.h);
            store_counters(a.counters, out_slot(a, ray), st.h);
            active = false;
        }
    }
}

template <int BLOCK, int MINB, bool SMEM_STACK>
__global__ void __launch_bounds__(BLOCK, MINB) batch_kernel(BatchArgs a) {
    extern __shared__ uint32_t smem[];
    DevScene* sc = reinterpret_cast<DevScene*>(smem);
    uint32_t* beg = reinterpret_cast<uint32_t*>(sc + a.S);
    {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(a.scenes);
        uint32_t* dst = reinterpret_cast<uint32_t*>(sc);
        const uint32_t words = a.S * uint32_t(sizeof(DevScene) / 4);
        for (uint32_t i = threadIdx.x; i < words; i += BLOCK) dst[i] = src[i];
        for (uint32_t i = threadIdx.x; i <= a.S; i += BLOCK) beg[i] = a.begin[i];
    }
    __syncthreads();
    uint32_t* stk_base = beg + ((a.S + 1 + 3) & ~3u);
    uint32_t lnode[SMEM_STACK ? 1 : MAX_LEVELS_ALL];
    float ltmax[SMEM_STACK ? 1 : MAX_LEVELS_ALL];
    uint32_t lcyc[SMEM_STACK ? 1 : CYC_WORDS];
    uint32_t* stkN;
    float* stkT;
    uint32_t* cyc;
    int stride;
    if (SMEM_STACK) {
        stkN = stk_base + threadIdx.x;
        stkT = reinterpret_cast<float*>(stk_base + a.maxL * BLOCK) + threadIdx.x;
        cyc = stk_base + 2 * a.maxL * BLOCK + threadIdx.x;
        stride = BLOCK;
    } else {
        stkN = lnode;
        stkT = ltmax;
        cyc = lcyc;
        stride = 1;
    }
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t n = ray_count(a);
    for (;;) {
        uint32_t t = 0;
        if (lane == 0) t = atomicAdd(a.work, 1u);
        t = __shfl_sync(0xFFFFFFFFu, t, 0);
        const uint64_t r0 = uint64_t(t) * a.K;
        if (r0 >= n) break;
        const uint32_t r1 = uint32_t(min(r0 + a.K, uint64_t(n)));
        for (uint32_t j = uint32_t(r0) + lane; j < r1; j += 32) {
            const uint32_t r = a.gather ? __ldg(a.gather + j) : j;
            const int lo = scene_of(beg, a.S, r);
            const float2* r2 = reinterpret_cast<const float2*>(a.rays + r);
            const float2 p = __ldg(r2), q = __ldg(r2 + 1), w = __ldg(r2 + 2);
            Hit h;
            // no budget: MAX_ITER + 1, which no cast reaches (the loop stops at MAX_ITER)
            if (!cast_ray_budget<false, !SMEM_STACK, true>(sc[lo], p.x, p.y, q.x, q.y, w.x, w.y, a.tmin, a.tmax, stkN, stkT,
                                                     cyc, stride, a.budget > 0 ? a.budget : MAX_ITER + 1, h)) {
                a.retry[atomicAdd(a.retry_n, 1u)] = r;
                continue;
            }
            store_hit(a.hits, out_slot(a, r), h);
            store_counters(a.counters, out_slot(a, r), h);
        }
    }
}

__host__ __device__ inline uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// Hit point and offset origin of a secondary ray: hp = o + normalize(d) * t
// (normalised exactly as the cast does), then hp + 1e-3 * n on the normal axis.
__device__ __forceinline__ bool secondary_origin(const vx_ray& r, const vx_hit& h, float org[3], int& axis,
                                                 float& sgn) {
    if (!(h.flags & VX_HIT_HIT)) return false;
    const float dd = (r.dx * r.dx + r.dy * r.dy) + r.dz * r.dz;
    const float inv = 1.0f / sqrtf(dd);
    org[0] = r.ox + (r.dx * inv) * h.t;
    org[1] = r.oy + (r.dy * inv) * h.t;
    org[2] = r.oz + (r.dz * inv) * h.t;
    axis = (h.flags >> 1) & 3;
    sgn = (h.flags & VX_HIT_NORMAL_NEG) ? -1.0f : 1.0f;
    org[axis] = org[axis] + sgn * 0.001f;
    return true;
}

// Bounce ray k (0 or 1) of primary ray i from its secondary origin: table
// direction j = mix64(seed ^ mix64(2i + k)) mod 4096, its z axis turned onto
// the hit normal.
__device__ __forceinline__ vx_ray bounce_ray(const float org[3], int axis, float sgn, uint64_t i, uint32_t k,
                                             uint64_t seed) {
    const uint32_t j = uint32_t(mix64(seed ^ mix64((i << 1) | k)) & (NUM_BOUNCE_DIRS - 1));
    const float u = g_bounce_dirs[3 * j], v = g_bounce_dirs[3 * j + 1], w = g_bounce_dirs[3 * j + 2] * sgn;
    vx_ray b;
    b.ox = org[0];
    b.oy = org[1];
    b.oz = org[2];
    if (axis == 0) { b.dx = w; b.dy = u; b.dz = v; }
    else if (axis == 1) { b.dx = v; b.dy = w; b.dz = u; }
    else { b.dx = u; b.dy = v; b.dz = w; }
    return b;
}

__global__ void spawn_bounce_kernel(const vx_ray* __restrict__ rays, const vx_hit* __restrict__ hits, uint32_t n,
                                    uint64_t seed, vx_ray* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const vx_ray r = rays[i];
    const vx_hit h = hits[i];
    float org[3];
    int axis;
    float sgn;
    if (!secondary_origin(r, h, org, axis, sgn)) {
        const vx_ray z{r.ox, r.oy, r.oz, 0.0f, 0.0f, 0.0f};
        out[2 * size_t(i)] = z;
        out[2 * size_t(i) + 1] = z;
        return;
    }
    for (uint32_t k = 0; k < 2; ++k) out[2 * size_t(i) + k] = bounce_ray(org, axis, sgn, i, k, seed);
}

__global__ void spawn_shadow_kernel(const vx_ray* __restrict__ rays, const vx_hit* __restrict__ hits, uint32_t n,
                                    float lx, float ly, float lz, vx_ray* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const vx_ray r = rays[i];
    const vx_hit h = hits[i];
    float org[3];
    int axis;
    float sgn;
    if (!secondary_origin(r, h, org, axis, sgn)) {
        out[i] = vx_ray{r.ox, r.oy, r.oz, 0.0f, 0.0f, 0.0f};
        return;
    }
    out[i] = vx_ray{org[0], org[1], org[2], lx, ly, lz};
}

// Bounce-ray compaction of a frame: the bounce pass casts only the 2 rays of
// every primary hit, grouped per scene by direction bin (rays that head the
// same way through the same scene take similar paths through the octree).
// A direction's bin is its octant and the order of its three axes by
// magnitude (8 x 6 = 48 bins).  The primary rays are split into chunks of at
// most COMPACT_CHUNK rays that never straddle a scene (chunk c: rays
// [start, end) of scene `scene`).  Per chunk and bin the bounce rays are
// counted; the counts become offsets per scene and bin; each chunk writes its
// bounce rays at their place with the hit slot (2i + k) of each in `map`.
// Order inside a (scene, bin) group: chunk by chunk, inside a chunk the first
// bounce rays (k = 0) of its primary rays in primary order, then the second
// ones.  Every position follows from the counts alone, so the order is the
// same on every run.
constexpr uint32_t COMPACT_CHUNK = 1024;
constexpr uint32_t NB = 48;  // direction bins

struct CompactChunk {
    uint32_t start, end, scene, pad;
};

__device__ __forceinline__ uint32_t bin_of(const vx_ray& r) {
    const uint32_t octant = uint32_t(r.dx > 0.0f) | (uint32_t(r.dy > 0.0f) << 1) | (uint32_t(r.dz > 0.0f) << 2);
    const float ax = fabsf(r.dx), ay = fabsf(r.dy), az = fabsf(r.dz);
    const uint32_t major = (ax >= ay && ax >= az) ? 0u : (ay >= az ? 1u : 2u);
    const uint32_t minor = (ax < ay && ax < az) ? 0u : (ay < az ? 1u : 2u);  // never equal to major
    const uint32_t next = major == 2u ? 0u : major + 1u;
    return octant * 6u + major * 2u + (minor == next ? 0u : 1u);
}

// Secondary origin of primary ray i, or false on a miss.
__device__ __forceinline__ bool bounce_origin(const vx_ray* __restrict__ rays, const vx_hit* __restrict__ hits,
                                              uint64_t i, float org[3], int& axis, float& sgn) {
    const vx_ray r = rays[i];
    const vx_hit h = hits[i];
    return secondary_origin(r, h, org, axis, sgn);
}

// counts[c * NB + b]: bounce rays of chunk c in bin b.
__global__ void __launch_bounds__(256) compact_count_kernel(const CompactChunk* __restrict__ chunks,
                                                            const vx_ray* __restrict__ rays,
                                                            const vx_hit* __restrict__ hits, uint64_t seed,
                                                            uint32_t* __restrict__ counts) {
    __shared__ uint32_t hist[NB];
    if (threadIdx.x < NB) hist[threadIdx.x] = 0;
    __syncthreads();
    const CompactChunk ch = chunks[blockIdx.x];
    for (uint32_t i = ch.start + threadIdx.x; i < ch.end; i += blockDim.x) {
        float org[3];
        int axis;
        float sgn;
        if (bounce_origin(rays, hits, i, org, axis, sgn)) {
            atomicAdd(&hist[bin_of(bounce_ray(org, axis, sgn, i, 0, seed))], 1u);
            atomicAdd(&hist[bin_of(bounce_ray(org, axis, sgn, i, 1, seed))], 1u);
        }
    }
    __syncthreads();
    if (threadIdx.x < NB) counts[blockIdx.x * NB + threadIdx.x] = hist[threadIdx.x];
}

// Block s: offs[c * NB + b] = bounce rays of scene s's bin b in its chunks
// before chunk c (an exclusive scan over the scene's chunks, one warp per
// bin, 32 chunks at a time); tot[s * NB + b] = the bin's total.
__global__ void __launch_bounds__(512) compact_scan_kernel(const uint32_t* __restrict__ counts,
                                                           const uint32_t* __restrict__ first_chunk,
                                                           uint32_t* __restrict__ offs, uint32_t* __restrict__ tot) {
    const uint32_t sc = blockIdx.x, lane = threadIdx.x & 31u, nwarps = blockDim.x >> 5;
    const uint32_t begin = first_chunk[sc], end = first_chunk[sc + 1];
    for (uint32_t b = threadIdx.x >> 5; b < NB; b += nwarps) {
        uint32_t run = 0;
        for (uint32_t c0 = begin; c0 < end; c0 += 32) {
            const uint32_t c = c0 + lane;
            const uint32_t v = c < end ? counts[c * NB + b] : 0u;
            uint32_t x = v;
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
                if (lane >= uint32_t(d)) x += y;
            }
            if (c < end) offs[c * NB + b] = run + (x - v);
            run += __shfl_sync(0xFFFFFFFFu, x, 31);
        }
        if (lane == 0) tot[sc * NB + b] = run;
    }
}

// One block: tot (S * NB totals in (scene, bin) order) becomes the exclusive
// prefix, the first compacted ray of each (scene, bin) group; cbegin[s] is
// scene s's first compacted ray and cbegin[S] the count.
__global__ void __launch_bounds__(1024) compact_base_kernel(uint32_t* __restrict__ tot, uint32_t S,
                                                            uint32_t* __restrict__ cbegin) {
    __shared__ uint32_t wsum[32];
    const uint32_t items = S * NB, per = (items + blockDim.x - 1) / blockDim.x;
    const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
    const uint32_t lo = min(items, t * per), hi = min(items, lo + per);
    uint32_t mine = 0;
    for (uint32_t j = lo; j < hi; ++j) mine += tot[j];
    uint32_t x = mine;  // inclusive scan over the block: warps, then warp totals
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
        if (lane >= uint32_t(d)) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        const uint32_t nw = blockDim.x >> 5;
        uint32_t w = lane < nw ? wsum[lane] : 0u;
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, d);
            if (lane >= uint32_t(d)) w += y;
        }
        wsum[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    uint32_t run = (warp ? wsum[warp - 1] : 0u) + (x - mine);
    for (uint32_t j = lo; j < hi; ++j) {
        const uint32_t v = tot[j];
        tot[j] = run;
        if (j % NB == 0) cbegin[j / NB] = run;
        run += v;
    }
    if (t == blockDim.x - 1) cbegin[S] = wsum[(blockDim.x >> 5) - 1];
}

// The record a cast writes for a zero-direction ray (cast_init: the ray fails
// validation before any scene data is read).
__device__ __forceinline__ void store_invalid(vx_hit* hits, uint64_t slot) {
    reinterpret_cast<uint4*>(hits)[slot] = make_uint4(0u, NONE, NONE, 0xFFFFu | (uint32_t(F_INVALID) << 16));
}

// Writes chunk c's bounce rays at base[scene * NB + b] + offs[c * NB + b] +
// their rank in the chunk's order (k = 0 rays in primary order, then k = 1);
// the slots of misses get the invalid record.  256 primary rays per round:
// lanes of one bin find each other with __match_any_sync and rank by lane,
// warp totals go through shared memory, a running count per bin crosses the
// rounds and the two k passes.
__global__ void __launch_bounds__(256) compact_scatter_kernel(const CompactChunk* __restrict__ chunks,
                                                              const vx_ray* __restrict__ rays,
                                                              const vx_hit* __restrict__ hits, uint64_t seed,
                                                              const uint32_t* __restrict__ offs,
                                                              const uint32_t* __restrict__ base,
                                                              vx_ray* __restrict__ out, uint32_t* __restrict__ map,
                                                              vx_hit* __restrict__ bounce_hits) {
    __shared__ uint32_t wcnt[8][NB];  // [warp][bin]
    __shared__ uint32_t run[NB];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t below = (1u << lane) - 1u;
    const CompactChunk ch = chunks[blockIdx.x];
    if (threadIdx.x < NB) run[threadIdx.x] = base[ch.scene * NB + threadIdx.x] + offs[blockIdx.x * NB + threadIdx.x];
    for (uint32_t k = 0; k < 2; ++k) {
        for (uint32_t r0 = ch.start; r0 < ch.end; r0 += 256) {
            for (uint32_t j = threadIdx.x; j < 8 * NB; j += blockDim.x) (&wcnt[0][0])[j] = 0u;
            __syncthreads();
            const uint32_t i = r0 + threadIdx.x;
            float org[3];
            int axis;
            float sgn;
            const bool hit = i < ch.end && bounce_origin(rays, hits, i, org, axis, sgn);
            vx_ray b{};
            uint32_t bin = NB;  // none
            if (hit) {
                b = bounce_ray(org, axis, sgn, i, k, seed);
                bin = bin_of(b);
            }
            const uint32_t peers = __match_any_sync(0xFFFFFFFFu, bin);
            if (hit && (peers & below) == 0) wcnt[warp][bin] = __popc(peers);  // the group's first lane
            __syncthreads();
            if (hit) {
                uint32_t p = run[bin] + __popc(peers & below);
                for (uint32_t w = 0; w < warp; ++w) p += wcnt[w][bin];
                out[p] = b;
                map[p] = 2 * i + k;
            } else if (k == 0 && i < ch.end) {
                store_invalid(bounce_hits, 2 * uint64_t(i));
                store_invalid(bounce_hits, 2 * uint64_t(i) + 1);
            }
            __syncthreads();
            if (threadIdx.x < NB) {
                uint32_t add = 0;
                for (uint32_t w = 0; w < 8; ++w) add += wcnt[w][threadIdx.x];
                run[threadIdx.x] += add;
            }
            __syncthreads();  // the next round clears wcnt
        }
    }
}

// Shadow-ray compaction (vx_cast_shadow_rays): one shadow ray per primary
// hit, in primary order.  Chunks of SHADOW_CHUNK primary rays: hits counted
// per chunk, counts scanned (the total is the device-side ray count of the
// cast), then each chunk writes its shadow rays at their offset with the
// primary index of each in `map`, and the invalid record into the slots of
// misses (what a cast writes for their zero-direction rays).
constexpr uint32_t SHADOW_CHUNK = 1024;

__device__ __forceinline__ bool hit_of(const vx_hit* hits, uint64_t i) {
    return (reinterpret_cast<const uint4*>(hits)[i].w >> 16) & VX_HIT_HIT;
}

__global__ void __launch_bounds__(256) shadow_count_kernel(const vx_hit* __restrict__ hits, uint32_t n,
                                                           uint32_t* __restrict__ counts) {
    __shared__ uint32_t part[8];
    uint32_t c = 0;
    for (uint32_t k = 0; k < 4; ++k) {
        const uint64_t i = uint64_t(blockIdx.x) * SHADOW_CHUNK + k * 256 + threadIdx.x;
        c += (i < n && hit_of(hits, i)) ? 1u : 0u;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xFFFFFFFFu, c, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < 8; ++w) t += part[w];
        counts[blockIdx.x] = t;
    }
}

// One block: exclusive scan of the nb chunk counts, 1,024 per round; *total
// receives the sum.
__global__ void __launch_bounds__(1024) shadow_scan_kernel(const uint32_t* __restrict__ counts, uint32_t nb,
                                                           uint32_t* __restrict__ offs, uint32_t* __restrict__ total) {
    __shared__ uint32_t wsum[32];
    __shared__ uint32_t carry;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < nb; base += 1024) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < nb ? counts[i] : 0u;
        uint32_t x = v;
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
            if (lane >= uint32_t(d)) x += y;
        }
        if (lane == 31) wsum[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = wsum[lane];
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, d);
                if (lane >= uint32_t(d)) w += y;
            }
            wsum[lane] = w;
        }
        __syncthreads();
        const uint32_t excl = carry + (warp ? wsum[warp - 1] : 0u) + (x - v);
        if (i < nb) offs[i] = excl;
        __syncthreads();
        if (threadIdx.x == 1023) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(256) shadow_scatter_kernel(const vx_ray* __restrict__ rays,
                                                             const vx_hit* __restrict__ hits, uint32_t n, float lx,
                                                             float ly, float lz, const uint32_t* __restrict__ offs,
                                                             vx_ray* __restrict__ out, uint32_t* __restrict__ map,
                                                             vx_hit* __restrict__ shadow_hits) {
    __shared__ uint32_t wcount[8];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t run = offs[blockIdx.x];
    for (uint32_t k = 0; k < 4; ++k) {
        const uint64_t i = uint64_t(blockIdx.x) * SHADOW_CHUNK + k * 256 + threadIdx.x;
        float org[3];
        int axis = 0;
        float sgn = 1.0f;
        bool hit = false;
        if (i < n) {
            const vx_ray r = rays[i];
            const vx_hit h = hits[i];
            hit = secondary_origin(r, h, org, axis, sgn);
        }
        const uint32_t bal = __ballot_sync(0xFFFFFFFFu, hit);
        if (lane == 0) wcount[warp] = __popc(bal);
        __syncthreads();
        uint32_t before = 0, round = 0;
        for (uint32_t w = 0; w < 8; ++w) {
            before += w < warp ? wcount[w] : 0u;
            round += wcount[w];
        }
        if (hit) {
            const uint32_t pos = run + before + __popc(bal & ((1u << lane) - 1u));
            out[pos] = vx_ray{org[0], org[1], org[2], lx, ly, lz};
            map[pos] = uint32_t(i);
        } else if (i < n) {
            store_invalid(shadow_hits, i);
        }
        run += round;
        __syncthreads();
    }
}

// The direction table (host), generated once: stratum-free cosine-weighted
// samples from a counter hash, evaluated in double and rounded to binary32.
const std::vector<float>& bounce_table() {
    static std::vector<float> tab = [] {
        std::vector<float> t(NUM_BOUNCE_DIRS * 3);
        for (uint32_t k = 0; k < NUM_BOUNCE_DIRS; ++k) {
            const uint64_t h1 = mix64(0xB0C0E5EEDULL + k), h2 = mix64(h1);
            const double u1 = double(h1 >> 11) * (1.0 / 9007199254740992.0);
            const double u2 = double(h2 >> 11) * (1.0 / 9007199254740992.0);
            const double rr = std::sqrt(u1), phi = 6.283185307179586476925 * u2;
            t[3 * k] = float(rr * std::cos(phi));
            t[3 * k + 1] = float(rr * std::sin(phi));
            t[3 * k + 2] = float(std::sqrt(std::max(0.0, 1.0 - u1)));
        }
        return t;
    }();
    return tab;
}

std::mutex g_table_mu;
bool g_table_ready[64] = {};

int ensure_bounce_table() {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(VX_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= 64) return fail(VX_EINVAL, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_table_mu);
    if (g_table_ready[dev]) return VX_OK;
    const auto& t = bounce_table();
    e = cudaMemcpyToSymbol(g_bounce_dirs, t.data(), t.size() * sizeof(float));
    if (e != cudaSuccess) return fail(VX_ECUDA, std::string("bounce table upload: ") + cudaGetErrorString(e));
    g_table_ready[dev] = true;
    return VX_OK;
}

struct Variant {
    int block;
    bool smem;
};

}  // namespace
}  // namespace vx

struct vx_batch {
    int device = 0;
    int per_sm[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // resident blocks per SM of each kernel variant (0 = unresolved)
    uint32_t S = 0;
    int maxL = 1;
    vx::DevScene* scenes = nullptr;  // device copy of the scene table
    uint32_t* work = nullptr;        // task counter (device scratch)
    uint32_t* retry = nullptr;       // budgeted tunings: set-aside count at [0], ray list from [64]
    uint64_t retry_cap = 0;          // rays the list holds
    vx_batch_tuning tuning{256, 32, 1, 0, 0};
    vx_batch_tuning bounce_tuning{0, 0, 0, 0, 0};  // block 0: the bounce pass of a frame uses `tuning`
    int num_sms = 148;
    cudaGraphExec_t frame = nullptr;
    cudaGraph_t frame_graph = nullptr;
    void* fscratch = nullptr;  // compacted frame: chunk counts and offsets, scene offsets, hit slots
    uint64_t fscratch_bytes = 0;
    // Buffers of the captured frame, for vx_batch_launch_frame_host and
    // vx_batch_frame_compaction.
    const vx_ray* f_primary = nullptr;
    vx_hit* f_primary_hits = nullptr;
    vx_hit* f_bounce_hits = nullptr;
    uint32_t f_n = 0;
    const uint32_t* f_cbegin = nullptr;  // compacted frame: S + 1 scene offsets of the compacted rays
    const uint32_t* f_map = nullptr;     // compacted frame: hit slot of each compacted ray
    cudaEvent_t ev_primary = nullptr;    // recorded inside the frame once the primary pass is done
    cudaEvent_t ev_copied = nullptr;
    cudaStream_t side = nullptr;         // copies the primary hits out while the bounce pass runs
    // A frame captured in parts (vx_batch_capture_frame_parts): part k is a
    // batch over the scenes of the frame's primary rays [r0, r1), with its own
    // compacted frame graph; `in` / `done` order its copies in and out.
    struct Part {
        vx_batch* sub;
        uint32_t r0, r1;
        cudaEvent_t in, done;
    };
    std::vector<Part> parts;
    uint32_t* part_begin = nullptr;  // device: the parts' scene offsets, relative to r0
    cudaStream_t in_stream = nullptr;  // copies the rays of the parts in
    cudaStream_t alt = nullptr;        // casts the odd parts (the even ones run on the caller's stream)
    cudaEvent_t ev_alt = nullptr;
};

namespace {

using vx::fail;

void forget_parts(vx_batch* b);

int cuda_err(cudaError_t e, const char* what) {
    return fail(VX_ECUDA, std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

size_t batch_smem(const vx_batch* b, bool smem_stack, int block) {
    size_t bytes = size_t(b->S) * sizeof(vx::DevScene) + ((size_t(b->S) + 1 + 3) & ~size_t(3)) * 4;
    if (smem_stack) bytes += (size_t(2) * size_t(b->maxL) + vx::CYC_WORDS) * size_t(block) * 4;
    return bytes;
}

template <int BLOCK, int MINB, bool SMEM, bool REFILL>
constexpr void (*batch_kernel_ptr())(vx::BatchArgs) {
    if constexpr (REFILL) return vx::batch_refill_kernel<BLOCK, MINB, SMEM>;
    else return vx::batch_kernel<BLOCK, MINB, SMEM>;
}

// Resolves (once per batch and variant, outside any stream capture) the
// dynamic shared-memory attribute and the resident blocks per SM.
template <int BLOCK, int MINB, bool SMEM, bool REFILL>
int prepare_variant(vx_batch* b, int slot) {
    if (b->per_sm[slot]) return VX_OK;
    auto kern = batch_kernel_ptr<BLOCK, MINB, SMEM, REFILL>();
    const size_t smem = batch_smem(b, SMEM, BLOCK);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return cuda_err(e, "vx_cast_batch: shared memory attribute");
    }
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BLOCK, smem);
    if (e != cudaSuccess) return cuda_err(e, "vx_cast_batch: occupancy");
    if (per_sm < 1) return fail(VX_EINVAL, "vx_cast_batch: kernel does not fit on an SM (too many scenes?)");
    b->per_sm[slot] = per_sm;
    return VX_OK;
}

template <int BLOCK, int MINB, bool SMEM, bool REFILL>
int launch_variant(vx_batch* b, int slot, const vx::BatchArgs& a, cudaStream_t st) {
    if (int r = prepare_variant<BLOCK, MINB, SMEM, REFILL>(b, slot)) return r;
    auto kern = batch_kernel_ptr<BLOCK, MINB, SMEM, REFILL>();
    kern<<<b->num_sms * b->per_sm[slot], BLOCK, batch_smem(b, SMEM, BLOCK), st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_err(e, "vx_cast_batch: launch");
    return VX_OK;
}

template <bool PREPARE_ONLY>
int dispatch_batch(vx_batch* b, const vx_batch_tuning& t, const vx::BatchArgs* a, cudaStream_t st) {
    const int slot = (t.block == 128 ? 0 : 4) + (t.stack_in_shared ? 0 : 2) + (t.refill ? 1 : 0);
#define VX_BATCH_CASE(SLOT, BLK, MINB, SMEM, REF)                                                      \
    case SLOT:                                                                                          \
        return PREPARE_ONLY ? prepare_variant<BLK, MINB, SMEM, REF>(b, SLOT)                            \
                            : launch_variant<BLK, MINB, SMEM, REF>(b, SLOT, *a, st);
    switch (slot) {
        VX_BATCH_CASE(0, 128, 6, true, false)
        VX_BATCH_CASE(1, 128, 4, true, true)
        VX_BATCH_CASE(2, 128, 6, false, false)
        VX_BATCH_CASE(3, 128, 4, false, true)
        VX_BATCH_CASE(4, 256, 3, true, false)
        VX_BATCH_CASE(5, 256, 2, true, true)
        VX_BATCH_CASE(6, 256, 3, false, false)
        VX_BATCH_CASE(7, 256, 2, false, true)
    }
#undef VX_BATCH_CASE
    return fail(VX_EINVAL, "vx_cast_batch: no kernel variant for this tuning");
}

int launch_batch(vx_batch* b, const vx_batch_tuning& t, const vx::BatchArgs& a, cudaStream_t st) {
    return dispatch_batch<false>(b, t, &a, st);
}

int prepare_batch(vx_batch* b, const vx_batch_tuning& t) { return dispatch_batch<true>(b, t, nullptr, nullptr); }

int check_tuning(const vx_batch_tuning* t) {
    if (!t || (t->block != 128 && t->block != 256) || t->rays_per_task < 32 || t->rays_per_task > 65536 ||
        (t->rays_per_task % 32) != 0 || t->refill < 0 || t->refill > 32 || t->budget < 0 || t->budget > 500 ||
        (t->budget && t->refill))
        return fail(VX_EINVAL, "batch tuning: block must be 128 or 256, rays_per_task a multiple of 32 in "
                               "[32, 65536], refill in [0, 32], budget in [0, 500] and 0 with refill");
    return VX_OK;
}

// The set-aside list of a budgeted tuning, for n rays.  Allocates (outside a
// stream capture only) when n grows.
int ensure_retry(vx_batch* b, uint64_t n, cudaStream_t st) {
    if (b->retry_cap >= n) return VX_OK;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (st) cudaStreamIsCapturing(st, &cs);
    if (cs != cudaStreamCaptureStatusNone)
        return fail(VX_EINVAL, "vx_cast_batch: a budgeted tuning needs its set-aside list before a capture "
                               "(cast once with at least this many rays first)");
    cudaFree(b->retry);
    b->retry = nullptr;
    b->retry_cap = 0;
    cudaError_t e = cudaMalloc(&b->retry, 256 + n * 4);
    if (e != cudaSuccess) return cuda_err(e, "vx_cast_batch: set-aside list");
    b->retry_cap = n;
    return VX_OK;
}

}  // namespace

extern "C" {

static int vx_batch_create_body(const vx_scene* const* scenes, uint32_t count, vx_batch** out) {
    if (!out || (!scenes && count) || count == 0 || count > 256)
        return fail(VX_EINVAL, "vx_batch_create: need 1..256 scenes");
    *out = nullptr;
    auto* b = new (std::nothrow) vx_batch();
    if (!b) return fail(VX_ENOMEM, "vx_batch_create: out of host memory");
    cudaGetDevice(&b->device);
    std::vector<vx::DevScene> host(count);
    for (uint32_t i = 0; i < count; ++i) {
        if (!scenes[i]) { delete b; return fail(VX_EINVAL, "vx_batch_create: null scene"); }
        if (vx::scene_device(scenes[i]) != b->device) {
            delete b;
            return fail(VX_EINVAL, "vx_batch_create: every scene must live on the current device");
        }
        host[i] = vx::scene_dev(scenes[i]);
        b->maxL = std::max(b->maxL, host[i].max_levels);
    }
    b->S = count;
    cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, b->device);
    cudaError_t e = cudaMalloc(&b->scenes, sizeof(vx::DevScene) * count);
    if (e == cudaSuccess) e = cudaMalloc(&b->work, 256);
    if (e == cudaSuccess) e = cudaMemcpy(b->scenes, host.data(), sizeof(vx::DevScene) * count, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(b->scenes);
        cudaFree(b->work);
        delete b;
        return cuda_err(e, "vx_batch_create");
    }
    *out = b;
    return VX_OK;
}

int vx_batch_create(const vx_scene* const* scenes, uint32_t count, vx_batch** out) {
    return vx::guarded("vx_batch_create", [&] { return vx_batch_create_body(scenes, count, out); });
}

int vx_batch_destroy(vx_batch* b) {
    if (!b) return VX_OK;
    forget_parts(b);
    if (b->in_stream) cudaStreamDestroy(b->in_stream);
    if (b->alt) cudaStreamDestroy(b->alt);
    if (b->ev_alt) cudaEventDestroy(b->ev_alt);
    if (b->frame) cudaGraphExecDestroy(b->frame);
    if (b->frame_graph) cudaGraphDestroy(b->frame_graph);
    if (b->ev_primary) cudaEventDestroy(b->ev_primary);
    if (b->ev_copied) cudaEventDestroy(b->ev_copied);
    if (b->side) cudaStreamDestroy(b->side);
    cudaFree(b->scenes);
    cudaFree(b->work);
    cudaFree(b->fscratch);
    cudaFree(b->retry);
    delete b;
    return VX_OK;
}

int vx_batch_set_tuning(vx_batch* b, const vx_batch_tuning* t) {
    if (!b) return fail(VX_EINVAL, "vx_batch_set_tuning: null batch");
    if (int r = check_tuning(t)) return r;
    b->tuning = *t;
    return VX_OK;
}

int vx_batch_get_tuning(const vx_batch* b, vx_batch_tuning* t) {
    if (!b || !t) return fail(VX_EINVAL, "vx_batch_get_tuning: null argument");
    *t = b->tuning;
    return VX_OK;
}

namespace {

int cast_batch_with(vx_batch* b, const vx_batch_tuning& t, const vx_ray* rays, const uint32_t* begin, uint32_t n,
                    float tmin, float tmax, vx_hit* hits, vx_ray_counters* counters, void* stream,
                    const uint32_t* map = nullptr, const uint32_t* n_dev = nullptr) {
    if (!b || !begin || (n && (!rays || !hits))) return fail(VX_EINVAL, "vx_cast_batch: null argument");
    if (reinterpret_cast<uintptr_t>(rays) % 8 || reinterpret_cast<uintptr_t>(hits) % 16 ||
        reinterpret_cast<uintptr_t>(counters) % 16 || reinterpret_cast<uintptr_t>(begin) % 4)
        return fail(VX_EINVAL, "vx_cast_batch: misaligned buffer");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(b->work, 0, 4, st);
    if (e != cudaSuccess) return cuda_err(e, "vx_cast_batch: reset work counter");
    if (n == 0) return VX_OK;
    vx::BatchArgs a{b->scenes, b->S, begin, rays, n, tmin, tmax, hits, counters, b->work,
                    uint32_t(t.rays_per_task), b->maxL, t.refill, map, n_dev};
    if (t.budget <= 0) return launch_batch(b, t, a, st);
    // Budgeted: the rays still running after t.budget iterations are set
    // aside, then a second launch casts them from the start.
    if (int r = ensure_retry(b, n, st)) return r;
    e = cudaMemsetAsync(b->retry, 0, 4, st);
    if (e != cudaSuccess) return cuda_err(e, "vx_cast_batch: reset set-aside count");
    a.budget = t.budget;
    a.retry = b->retry + 64;
    a.retry_n = b->retry;
    if (int r = launch_batch(b, t, a, st)) return r;
    e = cudaMemsetAsync(b->work, 0, 4, st);
    if (e != cudaSuccess) return cuda_err(e, "vx_cast_batch: reset work counter");
    vx::BatchArgs a2 = a;
    a2.budget = 0;
    a2.retry = nullptr;
    a2.retry_n = nullptr;
    a2.gather = b->retry + 64;
    a2.n_dev = b->retry;
    return launch_batch(b, t, a2, st);
}

const vx_batch_tuning& bounce_tuning_of(const vx_batch* b) {
    return b->bounce_tuning.block ? b->bounce_tuning : b->tuning;
}

}  // namespace

int vx_cast_batch(vx_batch* b, const vx_ray* rays, const uint32_t* begin, uint32_t n, float tmin, float tmax,
                  vx_hit* hits, vx_ray_counters* counters, void* stream) {
    if (!b) return fail(VX_EINVAL, "vx_cast_batch: null argument");
    return cast_batch_with(b, b->tuning, rays, begin, n, tmin, tmax, hits, counters, stream);
}

int vx_batch_set_bounce_tuning(vx_batch* b, const vx_batch_tuning* t) {
    if (!b) return fail(VX_EINVAL, "vx_batch_set_bounce_tuning: null batch");
    if (!t) { b->bounce_tuning = vx_batch_tuning{0, 0, 0, 0, 0}; return VX_OK; }
    if (int r = check_tuning(t)) return r;
    b->bounce_tuning = *t;
    return VX_OK;
}

static int vx_batch_autotune_body(vx_batch* b, const vx_ray* rays, const uint32_t* begin, uint32_t n, vx_hit* hits, void* stream,
                      vx_batch_tuning* best_out, float* best_ms_out) {
    if (!b || !begin || !rays || !hits || n == 0) return fail(VX_EINVAL, "vx_batch_autotune: bad argument");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    vx_batch_tuning bt = b->tuning;
    const int blocks[] = {128, 256};
    const int ks[] = {32, 64, 128, 256, 512, 1024};
    const int refills[] = {0, 8, 16, 24};
    const int budgets[] = {0, 32};
    if (int r = ensure_retry(b, n, st)) { cudaEventDestroy(e0); cudaEventDestroy(e1); return r; }
    for (int blk : blocks)
        for (int sm = 1; sm >= 0; --sm)
            for (int rf : refills)
                for (int bud : budgets)
                    for (int k : ks) {
                        if (rf && (k > 256 || bud)) continue;  // refilling warps draw rays one round at a time
                        vx_batch_tuning t{blk, k, sm, rf, bud};
                        float ms_min = 1e30f;
                        for (int rep = 0; rep < 3; ++rep) {
                            cudaEventRecord(e0, st);
                            int r = cast_batch_with(b, t, rays, begin, n, 0.0f, 3.402823466e+38f, hits, nullptr, st);
                            cudaEventRecord(e1, st);
                            if (r != VX_OK) { cudaEventDestroy(e0); cudaEventDestroy(e1); return r; }
                            cudaError_t e = cudaEventSynchronize(e1);
                            if (e != cudaSuccess) {
                                cudaEventDestroy(e0);
                                cudaEventDestroy(e1);
                                return cuda_err(e, "autotune");
                            }
                            float ms = 0;
                            cudaEventElapsedTime(&ms, e0, e1);
                            if (rep > 0) ms_min = std::min(ms_min, ms);
                        }
                        if (ms_min < best) { best = ms_min; bt = t; }
                    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->tuning = bt;
    if (best_out) *best_out = bt;
    if (best_ms_out) *best_ms_out = best;
    return VX_OK;
}

int vx_batch_autotune(vx_batch* b, const vx_ray* rays, const uint32_t* begin, uint32_t n, vx_hit* hits, void* stream,
                      vx_batch_tuning* best_out, float* best_ms_out) {
    return vx::guarded("vx_batch_autotune", [&] { return vx_batch_autotune_body(b, rays, begin, n, hits, stream, best_out, best_ms_out); });
}

int vx_bounce_table(float* out) {
    if (!out) return fail(VX_EINVAL, "vx_bounce_table: null argument");
    const auto& t = vx::bounce_table();
    std::copy(t.begin(), t.end(), out);
    return VX_OK;
}

int vx_spawn_bounce_rays(const vx_ray* rays, const vx_hit* hits, uint32_t n, uint64_t seed, vx_ray* out,
                         void* stream) {
    if (n && (!rays || !hits || !out)) return fail(VX_EINVAL, "vx_spawn_bounce_rays: null argument");
    if (int r = vx::ensure_bounce_table()) return r;
    if (n == 0) return VX_OK;
    vx::spawn_bounce_kernel<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(rays, hits, n, seed, out);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VX_OK : cuda_err(e, "vx_spawn_bounce_rays");
}

int vx_spawn_shadow_rays(const vx_ray* rays, const vx_hit* hits, uint32_t n, const float light_dir[3], vx_ray* out,
                         void* stream) {
    if (!light_dir || (n && (!rays || !hits || !out))) return fail(VX_EINVAL, "vx_spawn_shadow_rays: null argument");
    if (n == 0) return VX_OK;
    vx::spawn_shadow_kernel<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        rays, hits, n, light_dir[0], light_dir[1], light_dir[2], out);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VX_OK : cuda_err(e, "vx_spawn_shadow_rays");
}

}  // extern "C"

namespace vx {

uint64_t shadow_scratch_bytes(uint32_t n) {
    const uint64_t nb = (uint64_t(n) + SHADOW_CHUNK - 1) / SHADOW_CHUNK;
    auto a256 = [](uint64_t x) { return (x + 255) & ~uint64_t(255); };
    return a256(nb * 4) * 2 + 256 + a256(uint64_t(n) * 4) + a256(uint64_t(n) * sizeof(vx_ray));
}

int launch_shadow_compact(const vx_ray* rays, const vx_hit* hits, uint32_t n, const float light_dir[3], void* scratch,
                          vx_ray** out_rays, uint32_t** map, uint32_t** count, vx_hit* shadow_hits, void* stream) {
    const uint32_t nb = (n + SHADOW_CHUNK - 1) / SHADOW_CHUNK;
    auto a256 = [](uint64_t x) { return (x + 255) & ~uint64_t(255); };
    char* base = static_cast<char*>(scratch);
    uint32_t* counts = reinterpret_cast<uint32_t*>(base);
    uint32_t* offs = reinterpret_cast<uint32_t*>(base + a256(uint64_t(nb) * 4));
    *count = reinterpret_cast<uint32_t*>(base + 2 * a256(uint64_t(nb) * 4));
    *map = reinterpret_cast<uint32_t*>(base + 2 * a256(uint64_t(nb) * 4) + 256);
    *out_rays = reinterpret_cast<vx_ray*>(base + 2 * a256(uint64_t(nb) * 4) + 256 + a256(uint64_t(n) * 4));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    shadow_count_kernel<<<nb, 256, 0, st>>>(hits, n, counts);
    shadow_scan_kernel<<<1, 1024, 0, st>>>(counts, nb, offs, *count);
    shadow_scatter_kernel<<<nb, 256, 0, st>>>(rays, hits, n, light_dir[0], light_dir[1], light_dir[2], offs, *out_rays,
                                              *map, shadow_hits);
    return int(cudaGetLastError());
}

}  // namespace vx

namespace {

// The frame's events and side stream, created once per batch outside any capture.
int ensure_frame_events(vx_batch* b) {
    cudaError_t e = cudaSuccess;
    if (!b->ev_primary) e = cudaEventCreateWithFlags(&b->ev_primary, cudaEventDisableTiming);
    if (e == cudaSuccess && !b->ev_copied) e = cudaEventCreateWithFlags(&b->ev_copied, cudaEventDisableTiming);
    if (e == cudaSuccess && !b->side) e = cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking);
    return e == cudaSuccess ? VX_OK : cuda_err(e, "vx_batch: frame events");
}

// Inside a capture: an external event node that marks the end of the primary
// pass, so vx_batch_launch_frame_host can copy the primary hits out while the
// bounce pass runs.
int record_primary_done(vx_batch* b, cudaStream_t st) {
    cudaError_t e = cudaEventRecordWithFlags(b->ev_primary, st, cudaEventRecordExternal);
    return e == cudaSuccess ? VX_OK : cuda_err(e, "vx_batch: primary-pass event");
}

void forget_parts(vx_batch* b) {
    for (auto& p : b->parts) {
        vx_batch_destroy(p.sub);
        if (p.in) cudaEventDestroy(p.in);
        if (p.done) cudaEventDestroy(p.done);
    }
    b->parts.clear();
    cudaFree(b->part_begin);
    b->part_begin = nullptr;
}

void forget_frame(vx_batch* b) {
    if (b->frame) { cudaGraphExecDestroy(b->frame); b->frame = nullptr; }
    if (b->frame_graph) { cudaGraphDestroy(b->frame_graph); b->frame_graph = nullptr; }
    b->f_primary = nullptr;
    b->f_primary_hits = b->f_bounce_hits = nullptr;
    b->f_n = 0;
    b->f_cbegin = b->f_map = nullptr;
}

}  // namespace

extern "C" {

int vx_batch_capture_frame(vx_batch* b, const vx_ray* primary, const uint32_t* primary_begin, uint32_t n,
                           vx_hit* primary_hits, vx_ray* bounce, const uint32_t* bounce_begin, vx_hit* bounce_hits,
                           uint64_t seed, void* stream) {
    if (!b || !primary || !primary_begin || !primary_hits || !bounce || !bounce_begin || !bounce_hits || n == 0 ||
        n > 0x7FFFFFFFu)
        return fail(VX_EINVAL, "vx_batch_capture_frame: bad argument");
    if (int r = vx::ensure_bounce_table()) return r;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!st) return fail(VX_EINVAL, "vx_batch_capture_frame: capture needs a non-default stream");
    forget_parts(b);
    forget_frame(b);
    // Resolve shared-memory attributes and occupancy outside the capture.
    if (int r = prepare_batch(b, b->tuning)) return r;
    if (int r = prepare_batch(b, bounce_tuning_of(b))) return r;
    if (b->tuning.budget || bounce_tuning_of(b).budget)
        if (int r = ensure_retry(b, 2 * uint64_t(n), nullptr)) return r;
    if (int r = ensure_frame_events(b)) return r;
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_err(e, "vx_batch_capture_frame: begin capture");
    int r = vx_cast_batch(b, primary, primary_begin, n, 0.0f, 3.402823466e+38f, primary_hits, nullptr, stream);
    if (r == VX_OK) r = record_primary_done(b, st);
    if (r == VX_OK) r = vx_spawn_bounce_rays(primary, primary_hits, n, seed, bounce, stream);
    if (r == VX_OK)
        r = cast_batch_with(b, bounce_tuning_of(b), bounce, bounce_begin, 2 * n, 0.0f, 3.402823466e+38f, bounce_hits,
                            nullptr, stream);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(st, &g);
    if (r != VX_OK) { if (g) cudaGraphDestroy(g); return r; }
    if (e != cudaSuccess) return cuda_err(e, "vx_batch_capture_frame: end capture");
    e = cudaGraphInstantiate(&b->frame, g, 0);
    if (e != cudaSuccess) { cudaGraphDestroy(g); return cuda_err(e, "vx_batch_capture_frame: instantiate"); }
    b->frame_graph = g;
    b->f_primary = primary;
    b->f_primary_hits = primary_hits;
    b->f_bounce_hits = bounce_hits;
    b->f_n = n;
    return VX_OK;
}

// The compacted frame of batch b over primary rays [ray0, ray0 + n) of a
// frame: primary / primary_hits / bounce_hits are the frame's buffers (ray i
// of the frame at index i, its bounce slots at 2i, 2i + 1), primary_begin the
// S + 1 offsets of b's scenes relative to ray0, and bounce the part's own 2n
// rays of compaction output.  Bounce directions follow the frame index i, so
// a frame captured in parts casts the rays of the whole frame.
static int capture_compact(vx_batch* b, const vx_ray* primary, const uint32_t* primary_begin, uint32_t n,
                           vx_hit* primary_hits, vx_ray* bounce, vx_hit* bounce_hits, uint64_t seed, void* stream,
                           uint32_t ray0) {
    if (!b || !primary || !primary_begin || !primary_hits || !bounce || !bounce_hits || n == 0 || n > 0x7FFFFFFFu ||
        uint64_t(ray0) + n > 0x7FFFFFFFu)
        return fail(VX_EINVAL, "vx_batch_capture_frame_compact: bad argument");
    if (reinterpret_cast<uintptr_t>(bounce) % 8 || reinterpret_cast<uintptr_t>(bounce_hits) % 16 ||
        reinterpret_cast<uintptr_t>(primary_hits) % 16)
        return fail(VX_EINVAL, "vx_batch_capture_frame_compact: misaligned buffer");
    if (int r = vx::ensure_bounce_table()) return r;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!st) return fail(VX_EINVAL, "vx_batch_capture_frame_compact: capture needs a non-default stream");
    forget_frame(b);
    if (int r = prepare_batch(b, b->tuning)) return r;
    if (int r = prepare_batch(b, bounce_tuning_of(b))) return r;
    if (b->tuning.budget || bounce_tuning_of(b).budget)
        if (int r = ensure_retry(b, 2 * uint64_t(n), nullptr)) return r;
    if (int r = ensure_frame_events(b)) return r;
    // The chunk table follows the scene offsets, read once here: primary rays
    // of scene s are [begin[s], begin[s + 1]), split into chunks of at most
    // COMPACT_CHUNK rays.
    std::vector<uint32_t> hb(size_t(b->S) + 1);
    cudaError_t e = cudaMemcpyAsync(hb.data(), primary_begin, hb.size() * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_err(e, "vx_batch_capture_frame_compact: read scene offsets");
    if (hb[0] != 0 || hb[b->S] != n)
        return fail(VX_EINVAL, "vx_batch_capture_frame_compact: primary_begin must run from 0 to n");
    std::vector<vx::CompactChunk> chunks;
    std::vector<uint32_t> first(size_t(b->S) + 1, 0);
    for (uint32_t sc = 0; sc < b->S; ++sc) {
        if (hb[sc + 1] < hb[sc]) return fail(VX_EINVAL, "vx_batch_capture_frame_compact: primary_begin decreases");
        first[sc] = uint32_t(chunks.size());
        for (uint32_t a = hb[sc]; a < hb[sc + 1]; a += std::min(vx::COMPACT_CHUNK, hb[sc + 1] - a))
            chunks.push_back(
                vx::CompactChunk{ray0 + a, ray0 + a + std::min(vx::COMPACT_CHUNK, hb[sc + 1] - a), sc, 0u});
    }
    first[b->S] = uint32_t(chunks.size());
    const uint32_t nc = uint32_t(chunks.size());
    // Scratch (allocated outside the capture): chunk table, per-chunk bin
    // counts and offsets, first chunk of each scene, (scene, bin) totals and
    // then bases, the S + 1 scene offsets of the compacted rays and their 2n
    // hit slots.
    auto a256 = [](uint64_t x) { return (x + 255) & ~uint64_t(255); };
    const uint64_t o_cnt = a256(uint64_t(nc) * sizeof(vx::CompactChunk));
    const uint64_t o_offs = o_cnt + a256(uint64_t(nc) * vx::NB * 4), o_first = o_offs + a256(uint64_t(nc) * vx::NB * 4);
    const uint64_t o_tot = o_first + a256((uint64_t(b->S) + 1) * 4), o_cbeg = o_tot + a256(uint64_t(b->S) * vx::NB * 4);
    const uint64_t o_map = o_cbeg + a256((uint64_t(b->S) + 1) * 4), need = o_map + a256(uint64_t(n) * 8);
    if (need > b->fscratch_bytes) {
        cudaFree(b->fscratch);
        b->fscratch = nullptr;
        b->fscratch_bytes = 0;
        e = cudaMalloc(&b->fscratch, need);
        if (e != cudaSuccess) return cuda_err(e, "vx_batch_capture_frame_compact: scratch");
        b->fscratch_bytes = need;
    }
    char* base = static_cast<char*>(b->fscratch);
    auto* chunk_dev = reinterpret_cast<vx::CompactChunk*>(base);
    uint32_t* counts = reinterpret_cast<uint32_t*>(base + o_cnt);
    uint32_t* offs = reinterpret_cast<uint32_t*>(base + o_offs);
    uint32_t* first_dev = reinterpret_cast<uint32_t*>(base + o_first);
    uint32_t* tot = reinterpret_cast<uint32_t*>(base + o_tot);
    uint32_t* cbegin = reinterpret_cast<uint32_t*>(base + o_cbeg);
    uint32_t* map = reinterpret_cast<uint32_t*>(base + o_map);
    e = cudaMemcpyAsync(chunk_dev, chunks.data(), chunks.size() * sizeof(vx::CompactChunk), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(first_dev, first.data(), first.size() * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_err(e, "vx_batch_capture_frame_compact: chunk table");
    e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_err(e, "vx_batch_capture_frame_compact: begin capture");
    int r = vx_cast_batch(b, primary + ray0, primary_begin, n, 0.0f, 3.402823466e+38f, primary_hits + ray0, nullptr,
                          stream);
    if (r == VX_OK) r = record_primary_done(b, st);
    if (r == VX_OK) {
        vx::compact_count_kernel<<<nc, 256, 0, st>>>(chunk_dev, primary, primary_hits, seed, counts);
        vx::compact_scan_kernel<<<b->S, 512, 0, st>>>(counts, first_dev, offs, tot);
        vx::compact_base_kernel<<<1, 1024, 0, st>>>(tot, b->S, cbegin);
        vx::compact_scatter_kernel<<<nc, 256, 0, st>>>(chunk_dev, primary, primary_hits, seed, offs, tot, bounce, map,
                                                       bounce_hits);
        const cudaError_t le = cudaGetLastError();
        if (le != cudaSuccess) r = cuda_err(le, "vx_batch_capture_frame_compact: compaction launch");
    }
    if (r == VX_OK)
        r = cast_batch_with(b, bounce_tuning_of(b), bounce, cbegin, 2 * n, 0.0f, 3.402823466e+38f, bounce_hits,
                            nullptr, stream, map, cbegin + b->S);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(st, &g);
    if (r != VX_OK) { if (g) cudaGraphDestroy(g); return r; }
    if (e != cudaSuccess) return cuda_err(e, "vx_batch_capture_frame_compact: end capture");
    e = cudaGraphInstantiate(&b->frame, g, 0);
    if (e != cudaSuccess) { cudaGraphDestroy(g); return cuda_err(e, "vx_batch_capture_frame_compact: instantiate"); }
    b->frame_graph = g;
    b->f_primary = primary + ray0;
    b->f_primary_hits = primary_hits + ray0;
    b->f_bounce_hits = bounce_hits + 2 * size_t(ray0);
    b->f_n = n;
    b->f_cbegin = cbegin;
    b->f_map = map;
    return VX_OK;
}

int vx_batch_capture_frame_compact(vx_batch* b, const vx_ray* primary, const uint32_t* primary_begin, uint32_t n,
                                   vx_hit* primary_hits, vx_ray* bounce, vx_hit* bounce_hits, uint64_t seed,
                                   void* stream) {
    return vx::guarded("vx_batch_capture_frame_compact", [&] {
        if (b) forget_parts(b);
        return capture_compact(b, primary, primary_begin, n, primary_hits, bounce, bounce_hits, seed, stream, 0u);
    });
}

}  // extern "C"

namespace {

// Batch over scenes [s0, s0 + count) of b, with b's tunings.
int make_part(const vx_batch* b, uint32_t s0, uint32_t count, vx_batch** out) {
    *out = nullptr;
    auto* p = new (std::nothrow) vx_batch();
    if (!p) return fail(VX_ENOMEM, "vx_batch_capture_frame_parts: out of host memory");
    p->device = b->device;
    p->S = count;
    p->maxL = b->maxL;
    p->tuning = b->tuning;
    p->bounce_tuning = b->bounce_tuning;
    p->num_sms = b->num_sms;
    cudaError_t e = cudaMalloc(&p->scenes, sizeof(vx::DevScene) * count);
    if (e == cudaSuccess) e = cudaMalloc(&p->work, 256);
    if (e == cudaSuccess)
        e = cudaMemcpy(p->scenes, b->scenes + s0, sizeof(vx::DevScene) * count, cudaMemcpyDeviceToDevice);
    if (e != cudaSuccess) {
        vx_batch_destroy(p);
        return cuda_err(e, "vx_batch_capture_frame_parts: part");
    }
    *out = p;
    return VX_OK;
}

int capture_parts(vx_batch* b, const vx_ray* primary, const uint32_t* primary_begin, uint32_t n,
                  vx_hit* primary_hits, vx_ray* bounce, vx_hit* bounce_hits, uint64_t seed, uint32_t parts,
                  void* stream) {
    if (!b || !primary || !primary_begin || !primary_hits || !bounce || !bounce_hits || n == 0 || n > 0x7FFFFFFFu ||
        parts == 0)
        return fail(VX_EINVAL, "vx_batch_capture_frame_parts: bad argument");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!st) return fail(VX_EINVAL, "vx_batch_capture_frame_parts: capture needs a non-default stream");
    forget_parts(b);
    forget_frame(b);
    std::vector<uint32_t> hb(size_t(b->S) + 1);
    cudaError_t e = cudaMemcpyAsync(hb.data(), primary_begin, hb.size() * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_err(e, "vx_batch_capture_frame_parts: read scene offsets");
    if (hb[0] != 0 || hb[b->S] != n) return fail(VX_EINVAL, "vx_batch_capture_frame_parts: primary_begin must run from 0 to n");
    for (uint32_t sc = 0; sc < b->S; ++sc)
        if (hb[sc + 1] < hb[sc]) return fail(VX_EINVAL, "vx_batch_capture_frame_parts: primary_begin decreases");
    if (!b->in_stream) e = cudaStreamCreateWithFlags(&b->in_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess && !b->alt) e = cudaStreamCreateWithFlags(&b->alt, cudaStreamNonBlocking);
    if (e == cudaSuccess && !b->ev_alt) e = cudaEventCreateWithFlags(&b->ev_alt, cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_err(e, "vx_batch_capture_frame_parts: streams");
    if (int r = ensure_frame_events(b)) return r;
    // Part k: primary rays [k n / P, (k + 1) n / P) and the scenes they fall
    // in; its scene offsets are the frame's clamped to the part, relative to
    // its first ray.
    const uint32_t P = std::min(parts, n);
    std::vector<uint32_t> lb;
    struct Span { uint32_t r0, r1, s0, count, lb0; };
    std::vector<Span> spans;
    for (uint32_t k = 0; k < P; ++k) {
        const uint32_t r0 = uint32_t(uint64_t(n) * k / P), r1 = uint32_t(uint64_t(n) * (k + 1) / P);
        if (r1 == r0) continue;
        // scene of ray r: the last s with hb[s] <= r (hb[s + 1] > r)
        const uint32_t s0 = uint32_t(std::upper_bound(hb.begin(), hb.end(), r0) - hb.begin()) - 1;
        const uint32_t s1 = uint32_t(std::upper_bound(hb.begin(), hb.end(), r1 - 1) - hb.begin());
        spans.push_back(Span{r0, r1, s0, s1 - s0, uint32_t(lb.size())});
        for (uint32_t j = 0; j <= s1 - s0; ++j) lb.push_back(std::min(std::max(hb[s0 + j], r0), r1) - r0);
    }
    e = cudaMalloc(&b->part_begin, lb.size() * 4);
    if (e == cudaSuccess) e = cudaMemcpy(b->part_begin, lb.data(), lb.size() * 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_err(e, "vx_batch_capture_frame_parts: part offsets");
    for (const Span& sp : spans) {
        vx_batch::Part part{nullptr, sp.r0, sp.r1, nullptr, nullptr};
        int r = make_part(b, sp.s0, sp.count, &part.sub);
        if (r == VX_OK) {
            e = cudaEventCreateWithFlags(&part.in, cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&part.done, cudaEventDisableTiming);
            if (e != cudaSuccess) r = cuda_err(e, "vx_batch_capture_frame_parts: part events");
        }
        if (r == VX_OK)
            r = capture_compact(part.sub, primary, b->part_begin + sp.lb0, sp.r1 - sp.r0, primary_hits,
                                bounce + 2 * size_t(sp.r0), bounce_hits, seed, stream, sp.r0);
        b->parts.push_back(part);  // forget_parts releases whatever was made
        if (r != VX_OK) {
            forget_parts(b);
            return r;
        }
    }
    b->f_primary = primary;
    b->f_primary_hits = primary_hits;
    b->f_bounce_hits = bounce_hits;
    b->f_n = n;
    return VX_OK;
}

// The parts of a frame in order, part k on `st` for even k and on b->alt for
// odd k, so that the persistent kernels of one part fill the SMs the tail of
// the previous part leaves idle (the parts share no buffer or counter).  With
// host buffers (primary_host != null) the rays of every part first go in on
// the copy stream, part k casts once its rays are in, and its primary and
// bounce hits go out on the side stream once it is done, so that the copies
// of one part overlap the casts of its neighbours.  Returns after `st` has
// been made to wait for all of it (and, with host buffers, synchronised).
int run_parts(vx_batch* b, const vx_ray* primary_host, vx_hit* primary_hits_host, vx_hit* bounce_hits_host,
              cudaStream_t st) {
    const bool host = primary_host != nullptr;
    // every stream starts after whatever was queued on st before the call
    cudaError_t e = cudaEventRecord(b->ev_copied, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->alt, b->ev_copied, 0);
    if (host && e == cudaSuccess) e = cudaStreamWaitEvent(b->in_stream, b->ev_copied, 0);
    if (host && e == cudaSuccess) e = cudaStreamWaitEvent(b->side, b->ev_copied, 0);
    for (size_t k = 0; host && e == cudaSuccess && k < b->parts.size(); ++k) {
        const auto& p = b->parts[k];
        e = cudaMemcpyAsync(const_cast<vx_ray*>(b->f_primary) + p.r0, primary_host + p.r0,
                            size_t(p.r1 - p.r0) * sizeof(vx_ray), cudaMemcpyHostToDevice, b->in_stream);
        if (e == cudaSuccess) e = cudaEventRecord(p.in, b->in_stream);
    }
    for (size_t k = 0; e == cudaSuccess && k < b->parts.size(); ++k) {
        const auto& p = b->parts[k];
        cudaStream_t cs = (k & 1) ? b->alt : st;
        if (host) e = cudaStreamWaitEvent(cs, p.in, 0);
        if (e == cudaSuccess) e = cudaGraphLaunch(p.sub->frame, cs);
        if (e == cudaSuccess) e = cudaEventRecord(p.done, cs);
        if (!host) continue;
        if (e == cudaSuccess) e = cudaStreamWaitEvent(b->side, p.done, 0);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(primary_hits_host + p.r0, b->f_primary_hits + p.r0,
                                size_t(p.r1 - p.r0) * sizeof(vx_hit), cudaMemcpyDeviceToHost, b->side);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(bounce_hits_host + 2 * size_t(p.r0), b->f_bounce_hits + 2 * size_t(p.r0),
                                2 * size_t(p.r1 - p.r0) * sizeof(vx_hit), cudaMemcpyDeviceToHost, b->side);
    }
    if (e == cudaSuccess) e = cudaEventRecord(b->ev_alt, b->alt);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, b->ev_alt, 0);
    if (host) {
        if (e == cudaSuccess) e = cudaEventRecord(b->ev_copied, b->side);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(st, b->ev_copied, 0);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    return e == cudaSuccess ? VX_OK : cuda_err(e, host ? "vx_batch_launch_frame_host" : "vx_batch_launch_frame");
}

}  // namespace

extern "C" {

int vx_batch_capture_frame_parts(vx_batch* b, const vx_ray* primary, const uint32_t* primary_begin, uint32_t n,
                                 vx_hit* primary_hits, vx_ray* bounce, vx_hit* bounce_hits, uint64_t seed,
                                 uint32_t parts, void* stream) {
    return vx::guarded("vx_batch_capture_frame_parts", [&] {
        return capture_parts(b, primary, primary_begin, n, primary_hits, bounce, bounce_hits, seed, parts, stream);
    });
}

int vx_batch_launch_frame(vx_batch* b, void* stream) {
    if (b && !b->parts.empty()) return run_parts(b, nullptr, nullptr, nullptr, static_cast<cudaStream_t>(stream));
    if (!b || !b->frame) return fail(VX_EINVAL, "vx_batch_launch_frame: no captured frame");
    cudaError_t e = cudaGraphLaunch(b->frame, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? VX_OK : cuda_err(e, "vx_batch_launch_frame");
}

int vx_batch_launch_frame_host(vx_batch* b, const vx_ray* primary_host, vx_hit* primary_hits_host,
                               vx_hit* bounce_hits_host, void* stream) {
    if (b && !b->parts.empty()) {
        if (!primary_host || !primary_hits_host || !bounce_hits_host)
            return fail(VX_EINVAL, "vx_batch_launch_frame_host: null argument");
        return run_parts(b, primary_host, primary_hits_host, bounce_hits_host, static_cast<cudaStream_t>(stream));
    }
    if (!b || !b->frame) return fail(VX_EINVAL, "vx_batch_launch_frame_host: no captured frame");
    if (!primary_host || !primary_hits_host || !bounce_hits_host)
        return fail(VX_EINVAL, "vx_batch_launch_frame_host: null argument");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t n = b->f_n;
    // rays in; the frame; the primary hits out on the side stream as soon as
    // the frame's primary pass is done (while the bounce pass runs); the
    // bounce hits out after the frame; return when both copies are done.
    cudaError_t e = cudaMemcpyAsync(const_cast<vx_ray*>(b->f_primary), primary_host, n * sizeof(vx_ray),
                                    cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaGraphLaunch(b->frame, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->side, b->ev_primary, 0);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(primary_hits_host, b->f_primary_hits, n * sizeof(vx_hit), cudaMemcpyDeviceToHost, b->side);
    if (e == cudaSuccess) e = cudaEventRecord(b->ev_copied, b->side);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(bounce_hits_host, b->f_bounce_hits, 2 * n * sizeof(vx_hit), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, b->ev_copied, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e == cudaSuccess ? VX_OK : cuda_err(e, "vx_batch_launch_frame_host");
}

int vx_batch_frame_compaction(const vx_batch* b, uint32_t* scene_begin, uint32_t* map_host,
                              const uint32_t** cbegin_dev, const uint32_t** map_dev) {
    if (b && !b->parts.empty())
        return fail(VX_EINVAL, "vx_batch_frame_compaction: the frame was captured in parts (each part compacts its own rays)");
    if (!b || !b->frame || !b->f_cbegin)
        return fail(VX_EINVAL, "vx_batch_frame_compaction: no compacted frame captured");
    if (cbegin_dev) *cbegin_dev = b->f_cbegin;
    if (map_dev) *map_dev = b->f_map;
    if (scene_begin || map_host) {
        std::vector<uint32_t> sb(size_t(b->S) + 1);
        cudaError_t e = cudaMemcpy(sb.data(), b->f_cbegin, sb.size() * 4, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_err(e, "vx_batch_frame_compaction: read offsets");
        if (sb[b->S] > 2 * uint64_t(b->f_n)) return fail(VX_EINVAL, "vx_batch_frame_compaction: frame has not run");
        if (scene_begin) std::copy(sb.begin(), sb.end(), scene_begin);
        if (map_host && sb[b->S]) {
            e = cudaMemcpy(map_host, b->f_map, size_t(sb[b->S]) * 4, cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) return cuda_err(e, "vx_batch_frame_compaction: read slot map");
        }
    }
    return VX_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// vx_cast_batch_noalloc: the batched cast for callers that cannot allocate
// device memory, e.g. code running under a fixed device-memory budget owned by
// a host application, or on a frame path where cudaMalloc's implicit device
// synchronisation is not acceptable.  Its scratch (the task counter and the
// scene table) is the file-scope array below, VX_NOALLOC_SCRATCH_BYTES on
// every device that loads the library, held until the process exits.
// ---------------------------------------------------------------------------
namespace vx {
namespace {

constexpr uint32_t NOALLOC_TABLE_OFFSET = 256;  // the counter sits at offset 0
static_assert(NOALLOC_TABLE_OFFSET + VX_NOALLOC_MAX_SCENES * sizeof(DevScene) <= VX_NOALLOC_SCRATCH_BYTES,
              "no-alloc scratch too small for its scene table");
static __device__ __align__(256) unsigned char g_noalloc_scratch[VX_NOALLOC_SCRATCH_BYTES];

// The call's scene table travels as a kernel parameter (64 x 176 B, inside the
// 32 KB parameter limit of CUDA 12.1+), so staging it into the scratch is a
// stream-ordered kernel: no host-to-device copy from pageable memory, which
// would wait on the caller's stream.
struct NoallocTable {
    DevScene scene[VX_NOALLOC_MAX_SCENES];
    uint32_t count;
};
static_assert(sizeof(NoallocTable) <= 32000, "no-alloc scene table exceeds the kernel parameter space");

// One block: writes the first `count` table entries behind the counter and
// clears the counter (the previous call left its final value there).
__global__ void __launch_bounds__(256) noalloc_stage_kernel(const __grid_constant__ NoallocTable t,
                                                            unsigned char* scratch) {
    constexpr uint32_t WORDS = sizeof(DevScene) / 4;
    static_assert(sizeof(DevScene) % 4 == 0, "DevScene is copied word by word");
    const uint32_t* src = reinterpret_cast<const uint32_t*>(t.scene);
    uint32_t* dst = reinterpret_cast<uint32_t*>(scratch + NOALLOC_TABLE_OFFSET);
    for (uint32_t i = threadIdx.x; i < t.count * WORDS; i += blockDim.x) dst[i] = src[i];
    if (threadIdx.x == 0) *reinterpret_cast<uint32_t*>(scratch) = 0u;
}

struct NoallocDevice {
    bool ready = false;
    unsigned char* scratch = nullptr;  // device address of g_noalloc_scratch on this device
    int blocks = 0;                    // persistent grid size
};
std::mutex g_noalloc_mu;
NoallocDevice g_noalloc[64];

// Once per device, with that device current: resolve the scratch array's
// device address and the launch shape of the kernel variant used here.
int noalloc_setup(int dev, NoallocDevice*& out) {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    NoallocDevice& d = g_noalloc[dev];
    if (!d.ready) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_err(e, "vx_cast_batch_noalloc: cudaGetSymbolAddress");
        auto kern = batch_kernel<256, 3, true>;
        const size_t smem_max = size_t(VX_NOALLOC_MAX_SCENES) * sizeof(DevScene) +
                                ((size_t(VX_NOALLOC_MAX_SCENES) + 1 + 3) & ~size_t(3)) * 4 +
                                (size_t(2) * MAX_LEVELS_ALL + CYC_WORDS) * 256 * 4;
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem_max));
        if (e != cudaSuccess) return cuda_err(e, "vx_cast_batch_noalloc: shared memory attribute");
        int per_sm = 0, sms = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, smem_max);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return cuda_err(e, "vx_cast_batch_noalloc: occupancy");
        if (per_sm < 1) return fail(VX_EINVAL, "vx_cast_batch_noalloc: kernel does not fit on an SM");
        d.scratch = static_cast<unsigned char*>(ptr);
        d.blocks = per_sm * sms;
        d.ready = true;
    }
    out = &d;
    return VX_OK;
}

}  // namespace
}  // namespace vx

static int vx_cast_batch_noalloc_body(const vx_scene* const* scenes, uint32_t count, const vx_ray* rays,
                                     const uint32_t* begin, uint32_t n, float tmin, float tmax, vx_hit* hits,
                                     void* stream) {
    using namespace vx;
    if (!scenes || !begin || (n && (!rays || !hits))) return fail(VX_EINVAL, "vx_cast_batch_noalloc: null argument");
    if (count == 0 || count > VX_NOALLOC_MAX_SCENES)
        return fail(VX_EOVERFLOW, "vx_cast_batch_noalloc: scene count " + std::to_string(count) +
                                      " is outside 1.." + std::to_string(VX_NOALLOC_MAX_SCENES) +
                                      " (the size of its static scratch table)");
    if (reinterpret_cast<uintptr_t>(rays) % 8 || reinterpret_cast<uintptr_t>(hits) % 16 ||
        reinterpret_cast<uintptr_t>(begin) % 4)
        return fail(VX_EINVAL, "vx_cast_batch_noalloc: misaligned buffer");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_err(e, "vx_cast_batch_noalloc: cudaGetDevice");
    if (dev < 0 || dev >= 64) return fail(VX_EINVAL, "vx_cast_batch_noalloc: device ordinal out of range");
    NoallocTable table{};
    table.count = count;
    int maxL = 1;
    for (uint32_t i = 0; i < count; ++i) {
        if (!scenes[i]) return fail(VX_EINVAL, "vx_cast_batch_noalloc: null scene");
        if (scene_device(scenes[i]) != dev)
            return fail(VX_EINVAL, "vx_cast_batch_noalloc: every scene must live on the current device");
        table.scene[i] = scene_dev(scenes[i]);
        maxL = std::max(maxL, table.scene[i].max_levels);
    }
    NoallocDevice* d = nullptr;
    if (int r = noalloc_setup(dev, d)) return r;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // The scratch keeps the previous call's contents: rewrite the scene table
    // and clear the task counter on this call's stream.
    noalloc_stage_kernel<<<1, 256, 0, st>>>(table, d->scratch);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_err(e, "vx_cast_batch_noalloc: scratch staging");
    if (n == 0) return VX_OK;
    BatchArgs a{reinterpret_cast<const DevScene*>(d->scratch + NOALLOC_TABLE_OFFSET), count, begin, rays, n, tmin,
                tmax, hits, nullptr, reinterpret_cast<uint32_t*>(d->scratch), 32u, maxL};
    const size_t smem = size_t(count) * sizeof(DevScene) + ((size_t(count) + 1 + 3) & ~size_t(3)) * 4 +
                        (size_t(2) * size_t(maxL) + CYC_WORDS) * 256 * 4;
    batch_kernel<256, 3, true><<<d->blocks, 256, smem, st>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_err(e, "vx_cast_batch_noalloc: launch");
    return VX_OK;
}

extern "C" int vx_cast_batch_noalloc(const vx_scene* const* scenes, uint32_t count, const vx_ray* rays,
                                     const uint32_t* begin, uint32_t n, float tmin, float tmax, vx_hit* hits,
                                     void* stream) {
    return vx::guarded("vx_cast_batch_noalloc", [&] { return vx_cast_batch_noalloc_body(scenes, count, rays, begin, n, tmin, tmax, hits, stream); });
}

namespace vx {
VX_VIOLATION_READER(violations_batch)
}  // namespace vx
