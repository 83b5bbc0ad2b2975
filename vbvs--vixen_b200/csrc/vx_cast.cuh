// vx_cast.cuh - the ESVO cast of one ray, shared by every kernel that casts
// (vx_kernels.cu: plain and render; vx_batch.cu: persistent batched).
//
// One thread per ray.  The traversal restates LaineKarrasOctree::castRayImpl
// (SVO/src/SVOTraversal.cpp:516-691), handleLeafHit and the brick DDA
// (SVO/src/SVOBrickDDA.cpp:65-533) in IEEE binary32, compiled with
// --fmad=false and IEEE division / square root, so hit indices and t match
// the host code bit for bit.  Paths are relative to the reference project's
// VIXEN/ directory.
//
// Every floating-point value the reference computes is computed here by the
// same operations on the same operands.  What changes is only where it is
// computed: quantities that depend on the ray alone (the clamped ray-entry
// position, the slab reciprocals, the DDA step lengths, the ray-entry brick
// of the second lookup) are evaluated once per ray instead of at every leaf,
// voxel-corner t values are shared by the phases of one iteration that read
// them at the same position, and divisions by 8 and by 1 become the exact
// multiplications / identities they equal.
//
// Device layout (vx.h):
//   nodes      8 B per descriptor {child_ptr, valid | leaf << 8}; one 8-byte
//              load per parent change (the reference's fetchChildDescriptor)
//   grid       u32 per brick slot; read by the position-based brick lookups
//   occ        16 u32 per brick; one word per DDA step
//   rgba / dxt colour payload; one word / one 8-byte block per hit
// The per-ray ESVO stack (node, t_max per scale) lives in shared memory,
// [scale][thread] so neighbouring threads hit different banks.
#pragma once
#include <climits>
#include <cstdint>

#include "vx_dxtn.h"
#include "vx_internal.h"
#include "vx_raygen.h"

namespace vx {
namespace {

constexpr int ESVO_MAX_SCALE = 22;  // LaineKarrasOctree.h:337
constexpr int MAX_ITER = 500;       // SVOTraversal.cpp:588
#ifndef VX_CYCLE_START
#define VX_CYCLE_START 3
#endif
constexpr int CYCLE_START = VX_CYCLE_START;  // iteration from which loop states are compared
constexpr int CYC_WORDS = 16;                 // cycle-detection words per ray: two stored loop states
constexpr int LONG_FIRST = 16;                // first checkpoint of the long-cycle check (then 32, 64, ...)
constexpr int CK_WORDS = 16 + 2 * 23;         // long-cycle checkpoint: state, counters, stack (23 slots at most)
constexpr uint32_t SKIPPED = 1u << 31;        // in CastState::pushed: whole cycles were skipped
constexpr float FLT_MAX_ = 3.402823466e+38f;
constexpr uint32_t NONE = 0xFFFFFFFFu;

// Bounds-checked build (make checked -> libvx_checked.so, -DVX_CHECKED=1): every
// index into a scene array, the traversal stack and the batch's scene table is
// tested before its load; a failed test sets its bit in this translation
// unit's violation word (vx_bounds_checks reads and clears them) and the load
// uses index 0 instead.  The default build compiles no test.
#ifndef VX_CHECKED
#define VX_CHECKED 0
#endif
constexpr uint32_t V_NODE = 1u, V_GRID = 2u, V_BRICK = 4u, V_VOXEL = 8u, V_STACK = 16u, V_SCENE = 32u;
#if VX_CHECKED
static __device__ unsigned int vx_violation = 0u;
#endif
__device__ __forceinline__ uint32_t bounded(uint32_t i, uint32_t n, uint32_t code) {
#if VX_CHECKED
    if (i >= n) {
        atomicOr(&vx_violation, code);
        return 0u;
    }
#else
    (void)n;
    (void)code;
#endif
    return i;
}

constexpr uint32_t F_HIT = 1u;
constexpr uint32_t F_NEG = 1u << 3;
constexpr uint32_t F_ITER_CAP = 1u << 6;
constexpr uint32_t F_INVALID = 1u << 7;

// glm scalar min/max (func_common.inl): min = (y < x) ? y : x, max = (x < y) ? y : x.
__device__ __forceinline__ float gmin(float x, float y) { return (y < x) ? y : x; }
__device__ __forceinline__ float gmax(float x, float y) { return (x < y) ? y : x; }
__device__ __forceinline__ int imin(int x, int y) { return (y < x) ? y : x; }
__device__ __forceinline__ int imax(int x, int y) { return (x < y) ? y : x; }
__device__ __forceinline__ int iclamp(int v, int lo, int hi) { return imin(imax(v, lo), hi); }
__device__ __forceinline__ float fclamp(float v, float lo, float hi) { return gmin(gmax(v, lo), hi); }
__device__ __forceinline__ float min3(float a, float b, float c) { return gmin(gmin(a, b), c); }
__device__ __forceinline__ float max3(float a, float b, float c) { return gmax(gmax(a, b), c); }
// The same min / max where no operand is NaN or -0 (the octree loop's
// parametric t values and positions: finite, and every zero among them comes
// from x - x or a product of +0, so it is +0).  There glm's selections give
// the number the hardware min / max gives, in one instruction instead of a
// compare and a select.
__device__ __forceinline__ float nmin(float x, float y) { return fminf(x, y); }
__device__ __forceinline__ float nmax(float x, float y) { return fmaxf(x, y); }
__device__ __forceinline__ float nmin3(float a, float b, float c) { return fminf(fminf(a, b), c); }
__device__ __forceinline__ float nmax3(float a, float b, float c) { return fmaxf(fmaxf(a, b), c); }
__device__ __forceinline__ float nclamp(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }
// static_cast<int>(float) as x86-64 evaluates it (cvttss2si: INT_MIN when
// the value is outside the int range or NaN).
__device__ __forceinline__ int f2i(float f) {
    return (f >= -2147483648.0f && f < 2147483648.0f) ? __float2int_rz(f) : INT_MIN;
}
// The same for a value known to lie in [0, 2^31): the truncation alone.
__device__ __forceinline__ int f2i_in_range(float f) { return __float2int_rz(f); }

__device__ __forceinline__ uint32_t grid_lookup(const DevScene& s, int bx, int by, int bz) {
    // getBrickViewByGrid (SVOBuilder.h:107-116) over the dense table
    // (VoxelSceneCacher.cpp:670-713).  Every scene constructor keeps
    // bricks_per_axis <= 1024, so the index fits 32 bits.
    size_t li = uint32_t(bx) + uint32_t(s.bpa) * (uint32_t(by) + uint32_t(s.bpa) * uint32_t(bz));
#if VX_CHECKED
    const size_t slots = size_t(s.bpa) * size_t(s.bpa) * size_t(s.bpa);
    if (li >= slots || bx < 0 || by < 0 || bz < 0) { atomicOr(&vx_violation, V_GRID); li = 0; }
#endif
    return __ldg(s.grid + li);
}

struct Hit {
    float t;
    uint32_t brick, node, voxel, flags;
    uint32_t scale;                                   // RayHit::scale (0 on a miss)
    uint32_t iters, grid_reads, dda_steps;            // the reference traversal's counts
    uint32_t run_iters, run_grid_reads, run_dda_steps;  // what this kernel executed
};

// Per-ray constants of the brick stage.
struct RayB {
    float lo[3];     // ray origin in grid-local space: origin + (0 - worldMin)
    float d[3];      // normalised direction
    float inv[3];    // brick slab reciprocal, +-1e8 when |d| < 1e-8 (SVOBrickDDA.cpp:202-209)
    float tdel[3];   // DDA step length 1/|d|, FLT_MAX when |d| < 1e-8 (:424-430)
    int step[3];     // DDA step, 0 when |d| < 1e-8
};

// traverseBrickView (SVOBrickDDA.cpp:390-533) with brickVoxelSize = 1 and
// brickN = 8; occupancy from the brick's 512-bit mask.
__device__ __forceinline__ bool brick_dda(const DevScene& s, uint32_t brick, const float bmn[3], const RayB& rb,
                                          float tMin, float tMax, Hit& h) {
    int cur[3];
    float tNext[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float ep = rb.lo[a] + rb.d[a] * tMin;          // entryPoint
        cur[a] = iclamp(f2i(floorf(ep - bmn[a])), 0, 7);     // (entry - min) / 1
        if (fabsf(rb.d[a]) < 1e-8f) {
            tNext[a] = FLT_MAX_;
        } else if (rb.d[a] > 0.0f) {
            tNext[a] = tMin + ((bmn[a] + float(cur[a] + 1)) - ep) / rb.d[a];
        } else {
            tNext[a] = tMin + (ep - (bmn[a] + float(cur[a]))) / fabsf(rb.d[a]);
        }
    }
    const uint32_t* occ = reinterpret_cast<const uint32_t*>(s.occ) + size_t(bounded(brick, s.brick_count, V_BRICK)) * 16;
    for (int stepCount = 0; stepCount < 24; ++stepCount) {
        if (uint32_t(cur[0]) >= 8u || uint32_t(cur[1]) >= 8u || uint32_t(cur[2]) >= 8u) return false;
        ++h.dda_steps;
        const int vi = cur[2] * 64 + cur[1] * 8 + cur[0];
        const uint32_t word = __ldg(occ + (vi >> 5));
        if ((word >> (vi & 31)) & 1u) {
            float tn[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                if (fabsf(rb.d[a]) < 1e-8f) {
                    tn[a] = -__int_as_float(0x7f800000);
                } else {
                    // glm::min(t0, t1) of t0 = (vmn - lo) / d, t1 = ((vmn + 1) - lo) / d:
                    // rounded division by one divisor is monotone in the
                    // numerator, so the smaller is the near plane's quotient
                    // (t0 for d > 0, t1 for d < 0), and when the two round equal
                    // they are the same number.  No operand is NaN.
                    const float vmn = bmn[a] + float(cur[a]);
                    tn[a] = ((rb.d[a] > 0.0f ? vmn : vmn + 1.0f) - rb.lo[a]) / rb.d[a];
                }
            }
            float hitT = gmax(gmax(tn[0], tn[1]), tn[2]);
            hitT = gmax(hitT, 0.0f);
            int axis;
            if (tn[0] >= tn[1] && tn[0] >= tn[2]) axis = 0;
            else if (tn[1] >= tn[2]) axis = 1;
            else axis = 2;
            h.t = hitT;
            h.voxel = uint32_t(vi);
            const float dax = axis == 0 ? rb.d[0] : (axis == 1 ? rb.d[1] : rb.d[2]);
            h.flags |= F_HIT | (uint32_t(axis) << 1) | (dax > 0.0f ? F_NEG : 0u);
            return true;
        }
        if (tNext[0] < tNext[1] && tNext[0] < tNext[2]) {
            if (tNext[0] > tMax) return false;
            cur[0] += rb.step[0];
            tNext[0] += rb.tdel[0];
        } else if (tNext[1] < tNext[2]) {
            if (tNext[1] > tMax) return false;
            cur[1] += rb.step[1];
            tNext[1] += rb.tdel[1];
        } else {
            if (tNext[2] > tMax) return false;
            cur[2] += rb.step[2];
            tNext[2] += rb.tdel[2];
        }
    }
    return false;
}

struct Coef {
    float tx_coef, ty_coef, tz_coef, tx_bias, ty_bias, tz_bias;
    int octant_mask;
};

// Everything castRayImpl carries from one loop iteration to the next, plus the
// per-ray constants the iterations read.  cast_init fills it (the part of
// castRayImpl before the loop); every cast_step runs one loop iteration.
struct CastState {
    Hit h;
    // per-ray constants
    float ox, oy, oz, dx, dy, dz, tEntry;
    float tRayStart;       // world t where the octree walk starts (SVOTraversal.cpp:545)
    Coef c;
    float rlx, rly, rlz;   // clamped ray-entry position in [0,1] (SVOBrickDDA.cpp:107-109)
    RayB rb;
    uint32_t brick2;       // ray-entry brick of the second lookup, read on first use
    bool have_brick2;
    // loop state (ESVOTraversalState, LaineKarrasOctree.h:229-257)
    int scale, idx, iter;
    uint32_t parent;
    bool fetched;
    float px, py, pz, scale_exp2, t_min, t_max, hh;
    // the parent's descriptor: child pointer and valid | leaf << 8 in world
    // octant order.  The reference tests the mirrored masks (mirrorMask,
    // SVOTypes.h:343-364, moves bit i to i ^ flip, flip = ~octant_mask & 7) at
    // the ray-space octant idx; that is bit idx ^ flip of the unmirrored mask.
    uint32_t pChild, pMask;
    uint32_t pushed;       // stack slots written by PUSH (bit scale - minScale); bit 31: SKIPPED
    float t_root;          // t_max of the unwritten slots
    // cycle detection
    uint32_t d1g, d1d;     // grid reads / DDA steps of the previous iteration
    uint32_t sig1, sig2;   // signatures of the loop states one and two iterations back
    uint32_t ck_sig;       // signature of the long-cycle checkpoint
    int cand_p, cand_at;   // deferred check: pending candidate's period, iteration it is confirmed at
};

__device__ __forceinline__ void cast_finish(CastState& st) {
    st.h.iters = uint32_t(st.iter);
    st.h.run_iters = st.h.iters;
    st.h.run_grid_reads = st.h.grid_reads;
    st.h.run_dda_steps = st.h.dda_steps;
    if (st.iter >= MAX_ITER) st.h.flags |= F_ITER_CAP;
}

// LODParameters (SVO/include/SVOLOD.h:50-177): ray-cone diameter at the
// origin and its growth per unit distance.
struct LodCone {
    float orig, dir;
};

// castRayImpl up to its loop (SVOTraversal.cpp:516-586).  Returns true when the
// ray is already finished (invalid input or no overlap with the world box).
__device__ __forceinline__ bool cast_init(const DevScene& s, float ox, float oy, float oz, float ddx, float ddy,
                                          float ddz, float tMinArg, float tMaxArg, uint32_t* stkN, float* stkT,
                                          int stride, CastState& st) {
    Hit& h = st.h;
    h.t = 0.0f;
    h.brick = NONE;
    h.node = NONE;
    h.voxel = 0xFFFFu;
    h.flags = 0;
    h.scale = 0;
    h.iters = 0;
    h.grid_reads = 0;
    h.dda_steps = 0;
    h.run_iters = 0;
    h.run_grid_reads = 0;
    h.run_dda_steps = 0;
    // validateRayInput (:238-259)
    if (s.node_count == 0) { h.flags = F_INVALID; return true; }
    float dx, dy, dz;
    {
        const float dd = (ddx * ddx + ddy * ddy) + ddz * ddz;
        const float inv = 1.0f / sqrtf(dd);
        dx = ddx * inv; dy = ddy * inv; dz = ddz * inv;
        // length(normalize(d)) < 1e-6: for dd in [1e-30, 1e30] every component is
        // finite and the normalised length is 1 within a few ulp, so the check
        // can only fail outside that range.  In that range |d_i| <= sqrt(dd),
        // so the normalised components are finite as well and only the origin
        // needs the isnan || isinf test; outside it (an infinite or NaN input
        // lands there too) the components are tested.
        // isnan || isinf of a value: !(|x| < inf) is both tests at once
        const float inf = __int_as_float(0x7F800000);
        if (!(dd >= 1e-30f && dd <= 1e30f)) {
            const float len = sqrtf((dx * dx + dy * dy) + dz * dz);
            if (len < 1e-6f || !(fabsf(dx) < inf) || !(fabsf(dy) < inf) || !(fabsf(dz) < inf)) {
                h.flags = F_INVALID;
                return true;
            }
        }
        if (!(fabsf(ox) < inf) || !(fabsf(oy) < inf) || !(fabsf(oz) < inf)) {
            h.flags = F_INVALID;
            return true;
        }
    }
    const float wminx = s.wmin[0], wminy = s.wmin[1], wminz = s.wmin[2];
    const bool inside = ox >= wminx && ox <= s.wmax[0] && oy >= wminy && oy <= s.wmax[1] && oz >= wminz &&
                        oz <= s.wmax[2];
    // 1/d per axis, the one division every reciprocal below derives from:
    // 1/(-|d|) = -|1/d| and 1/|d| = |1/d| exactly (IEEE division is symmetric
    // in sign), so intersectAABB, computeRayCoefficients and the brick DDA
    // reciprocals need no further division.
    const float rcp[3] = {1.0f / dx, 1.0f / dy, 1.0f / dz};
    // intersectAABB (:117-149)
    float tEntry, tExit;
    {
        const float o[3] = {ox, oy, oz}, d[3] = {dx, dy, dz};
        float tnear[3], tfar[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            float inv;
            if (fabsf(d[i]) < 1e-8f) {
                if (o[i] < s.wmin[i] || o[i] > s.wmax[i]) return true;
                inv = (d[i] >= 0.0f) ? 1e20f : -1e20f;
            } else {
                inv = rcp[i];
            }
            // glm::min / max of the two plane t values: multiplication by one
            // factor is monotone, so their order is the sign of inv (equal
            // values are the same number); neither is NaN
            const float t0 = (s.wmin[i] - o[i]) * inv;
            const float t1 = (s.wmax[i] - o[i]) * inv;
            const bool pos = inv > 0.0f;
            tnear[i] = pos ? t0 : t1;
            tfar[i] = pos ? t1 : t0;
        }
        tEntry = max3(tnear[0], tnear[1], tnear[2]);
        tExit = min3(tfar[0], tfar[1], tfar[2]);
        if (!(tEntry <= tExit && tExit >= 0.0f)) return true;
    }
    tEntry = gmax(tEntry, tMinArg);
    tExit = gmin(tExit, tMaxArg);
    if (tEntry >= tExit || tExit < 0.0f) return true;
    const float tRayStart = inside ? 0.0f : gmax(0.0f, tEntry);
    // x / size, as a product where 1 / size is exact (a power-of-two size):
    // both round the same real number once.
    auto by_size = [&](float x, int i) { return s.wsinv[i] != 0.0f ? x * s.wsinv[i] : x / s.wsize[i]; };
    const float nox = by_size(ox + dx * tRayStart - wminx, 0) + 1.0f;
    const float noy = by_size(oy + dy * tRayStart - wminy, 1) + 1.0f;
    const float noz = by_size(oz + dz * tRayStart - wminz, 2) + 1.0f;
    // computeRayCoefficients (:699-728)
    Coef& c = st.c;
    {
        // t_coef = 1 / -|d|, with |d| raised to 1e-5 (copysign) below that
        const float k_small = 1.0f / -1e-5f;
        c.tx_coef = fabsf(dx) < 1e-5f ? k_small : -fabsf(rcp[0]);
        c.ty_coef = fabsf(dy) < 1e-5f ? k_small : -fabsf(rcp[1]);
        c.tz_coef = fabsf(dz) < 1e-5f ? k_small : -fabsf(rcp[2]);
        c.tx_bias = c.tx_coef * nox;
        c.ty_bias = c.ty_coef * noy;
        c.tz_bias = c.tz_coef * noz;
        c.octant_mask = 7;
        if (dx > 0.0f) { c.octant_mask ^= 1; c.tx_bias = 3.0f * c.tx_coef - c.tx_bias; }
        if (dy > 0.0f) { c.octant_mask ^= 2; c.ty_bias = 3.0f * c.ty_coef - c.ty_bias; }
        if (dz > 0.0f) { c.octant_mask ^= 4; c.tz_bias = 3.0f * c.tz_coef - c.tz_bias; }
    }
    float t_min, t_max;
    if (inside) {
        t_min = 0.0f;
        t_max = min3(c.tx_coef - c.tx_bias, c.ty_coef - c.ty_bias, c.tz_coef - c.tz_bias);
        t_max = gmin(t_max, 1.0f);
    } else {
        t_min = max3(2.0f * c.tx_coef - c.tx_bias, 2.0f * c.ty_coef - c.ty_bias, 2.0f * c.tz_coef - c.tz_bias);
        t_max = min3(c.tx_coef - c.tx_bias, c.ty_coef - c.ty_bias, c.tz_coef - c.tz_bias);
        t_min = gmax(t_min, 0.0f);
        t_max = gmin(t_max, 1.0f);
    }
    // initializeTraversalState (:261-280): stack[minScale..22] = (root, t_max).
    // Kept implicitly: a slot not yet pushed (bit clear in `pushed`) reads as
    // (0, t_root), so no slot is written here.
    st.pushed = 0u;
    st.t_root = t_max;
    int idx = 0;
    float px = 1.0f, py = 1.0f, pz = 1.0f;
    const bool csx = fabsf(dx) >= 1e-5f, csy = fabsf(dy) >= 1e-5f, csz = fabsf(dz) >= 1e-5f;
    // selectInitialOctant (:730-766)
    {
        const bool usePos = (t_min < 0.01f);
        const float mx = (c.octant_mask & 1) ? nox : (3.0f - nox);
        const float my = (c.octant_mask & 2) ? noy : (3.0f - noy);
        const float mz = (c.octant_mask & 4) ? noz : (3.0f - noz);
        if (!csx || usePos) { if (mx >= 1.5f) { idx |= 1; px = 1.5f; } }
        else if (1.5f * c.tx_coef - c.tx_bias > t_min) { idx ^= 1; px = 1.5f; }
        if (!csy || usePos) { if (my >= 1.5f) { idx |= 2; py = 1.5f; } }
        else if (1.5f * c.ty_coef - c.ty_bias > t_min) { idx ^= 2; py = 1.5f; }
        if (!csz || usePos) { if (mz >= 1.5f) { idx |= 4; pz = 1.5f; } }
        else if (1.5f * c.tz_coef - c.tz_bias > t_min) { idx ^= 4; pz = 1.5f; }
    }
    // handleLeafHit quantities that depend on the ray only (SVOBrickDDA.cpp:98-121, 140-143, 165-166)
    const float te0 = gmax(tEntry, 0.0f);
    st.rlx = fclamp(by_size((ox + dx * te0) - wminx, 0), 0.001f, 0.999f);
    st.rly = fclamp(by_size((oy + dy * te0) - wminy, 1), 0.001f, 0.999f);
    st.rlz = fclamp(by_size((oz + dz * te0) - wminz, 2), 0.001f, 0.999f);
    RayB& rb = st.rb;
    rb.lo[0] = ox + (0.0f - wminx);
    rb.lo[1] = oy + (0.0f - wminy);
    rb.lo[2] = oz + (0.0f - wminz);
    rb.d[0] = dx; rb.d[1] = dy; rb.d[2] = dz;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        rb.inv[i] = (fabsf(rb.d[i]) < 1e-8f) ? ((rb.d[i] >= 0) ? 1e8f : -1e8f) : rcp[i];
        rb.tdel[i] = (fabsf(rb.d[i]) < 1e-8f) ? FLT_MAX_ : fabsf(rcp[i]);
        rb.step[i] = (fabsf(rb.d[i]) < 1e-8f) ? 0 : ((rb.d[i] > 0.0f) ? 1 : -1);
    }
    st.ox = ox; st.oy = oy; st.oz = oz;
    st.dx = dx; st.dy = dy; st.dz = dz;
    st.tEntry = tEntry;
    st.tRayStart = tRayStart;
    st.brick2 = 0;
    st.have_brick2 = false;
    st.scale = ESVO_MAX_SCALE;
    st.idx = idx;
    st.iter = 0;
    st.parent = 0;
    st.fetched = false;
    st.px = px; st.py = py; st.pz = pz;
    st.scale_exp2 = 0.5f;
    st.t_min = t_min;
    st.t_max = t_max;
    st.hh = t_max;
    st.pChild = st.pMask = 0;
    st.d1g = st.d1d = 0;
    st.sig1 = st.sig2 = st.ck_sig = 0;
    st.cand_p = st.cand_at = 0;
    return false;
}

// One iteration of castRayImpl's loop (SVOTraversal.cpp:597-688) is built
// from the parts below: the corner t values, the leaf stage (handleLeafHit and
// the brick DDA), ADVANCE + POP, and the end-of-iteration cycle check; each
// reads and writes only CastState.
//
// Cycle detection: the loop state (scale, idx, fetched, parent, pos, t_min,
// t_max, h) with the stack determines every later iteration, and a cycle only
// rewrites stack slots with the values they already hold.  So once the state
// repeats after one or two iterations the ray can neither hit nor leave before
// the 500-iteration cap: the result is the capped miss and the remaining
// iterations' counters repeat the cycle's.  From iteration CYCLE_START on,
// every state gets a 32-bit signature, and the signatures of the two previous
// states stay in registers; equal states always have equal signatures.  Every
// iteration from CYCLE_START that does not end the ray records one, so at
// iteration i the signature one back exists from CYCLE_START + 1 and the one
// two back from CYCLE_START + 2.  Two
// policies, the same results:
//  - immediate (DEFER = false; the stack in shared memory): every state is
//    stored in one of two parity slots (cyc[(p * 8 + k) * stride]), and a
//    signature equal to the one 1 or 2 iterations back compares the stored
//    state word by word, so the repeat ends the ray on the iteration it occurs;
//  - deferred (DEFER = true; the stack in local memory, where a store per
//    iteration costs more): a signature match makes the state a candidate,
//    stored once, and the state p iterations later is compared with it;
//    equal states prove the repeat, unequal ones drop the candidate, so a
//    repeat ends the ray at most p iterations later.
// With LOD the cut test reads only the loop state and per-ray constants, so a
// repeating state still cannot end.
//
// LOD: castRayWithLOD (SVOTraversal.cpp:198-232) with LODParameters `lod`
// (enabled, lod.dir > 0): the termination test of :613-651 runs on every
// processed child before the leaf test.

// Voxel corners at the iteration's position (computeVoxelCorners, :786-794)
// and the corrected tc_max (:768-784); checkChildValidity, PUSH and ADVANCE
// all evaluate them at this position and t_max.
struct Corners {
    float tx, ty, tz, tcc;
};
__device__ __forceinline__ Corners corners_of(const CastState& st, bool csx, bool csy, bool csz) {
    const Coef& c = st.c;
    Corners k;
    k.tx = st.px * c.tx_coef - c.tx_bias;
    k.ty = st.py * c.ty_coef - c.ty_bias;
    k.tz = st.pz * c.tz_coef - c.tz_bias;
    k.tcc = nmin3((csx && fabsf(k.tx) < 1000.0f) ? k.tx : st.t_max, (csy && fabsf(k.ty) < 1000.0f) ? k.ty : st.t_max,
                  (csz && fabsf(k.tz) < 1000.0f) ? k.tz : st.t_max);
    return k;
}

// handleLeafHit (SVOBrickDDA.cpp:65-181) and traverseBrickAndReturnHit
// (:187-225) at the iteration's leaf child; true (and the hit record
// complete) when the brick DDA hits.
__device__ __forceinline__ bool leaf_stage(const DevScene& s, CastState& st, bool csx, bool csy, bool csz) {
    Hit& h = st.h;
    const Coef& c = st.c;
    float lx = st.px, ly = st.py, lz = st.pz;
    if ((c.octant_mask & 1) == 0) lx = 3.0f - st.scale_exp2 - lx;
    if ((c.octant_mask & 2) == 0) ly = 3.0f - st.scale_exp2 - ly;
    if ((c.octant_mask & 4) == 0) lz = 3.0f - st.scale_exp2 - lz;
    const float ix = nclamp(csx ? (lx - 1.0f) + ((st.dx > 0) ? 0.001f : -0.001f) : st.rlx, 0.001f, 0.999f);
    const float iy = nclamp(csy ? (ly - 1.0f) + ((st.dy > 0) ? 0.001f : -0.001f) : st.rly, 0.001f, 0.999f);
    const float iz = nclamp(csz ? (lz - 1.0f) + ((st.dz > 0) ? 0.001f : -0.001f) : st.rlz, 0.001f, 0.999f);
    const int bmax = s.bpa - 1;
    // Method 1: ESVO state position (x / 8 == x * 0.125 exactly)
    const float hx = nclamp(ix * s.wsize[0], 0.0f, s.wsm[0]);
    const float hy = nclamp(iy * s.wsize[1], 0.0f, s.wsm[1]);
    const float hz = nclamp(iz * s.wsize[2], 0.0f, s.wsm[2]);
    // hx, hy, hz are clamped to [0, wsize - 0.001]: the conversions are in range
    uint32_t brick = grid_lookup(s, iclamp(f2i_in_range(hx * 0.125f), 0, bmax),
                                 iclamp(f2i_in_range(hy * 0.125f), 0, bmax), iclamp(f2i_in_range(hz * 0.125f), 0, bmax));
    ++h.grid_reads;
    uint32_t method = 1;
    if (brick == NONE) {
        // Method 2: ray entry position (the same brick for the whole ray)
        if (!st.have_brick2) {
            const float te0 = gmax(st.tEntry, 0.0f);
            const float ex = fclamp(((st.ox + st.dx * te0) - s.wmin[0]) + st.dx * 0.01f, 0.0f, s.wsm[0]);
            const float ey = fclamp(((st.oy + st.dy * te0) - s.wmin[1]) + st.dy * 0.01f, 0.0f, s.wsm[1]);
            const float ez = fclamp(((st.oz + st.dz * te0) - s.wmin[2]) + st.dz * 0.01f, 0.0f, s.wsm[2]);
            st.brick2 = grid_lookup(s, iclamp(f2i_in_range(ex * 0.125f), 0, bmax),
                                    iclamp(f2i_in_range(ey * 0.125f), 0, bmax),
                                    iclamp(f2i_in_range(ez * 0.125f), 0, bmax));
            st.have_brick2 = true;
        }
        brick = st.brick2;
        ++h.grid_reads;
        method = 2;
    }
    if (brick == NONE) {
        // Fallback 3: leaf child of the parent at the local octant
        // (leafToBrickView, SVORebuild.cpp:569-574)
        method = 3;
        const uint32_t lo = uint32_t(st.idx ^ (~c.octant_mask & 7));
        const uint32_t valid = st.pMask & 0xFFu, leafs = valid & (st.pMask >> 8);
        if ((leafs >> lo) & 1u) {
            const uint32_t ci = st.pChild + __popc(valid & ~leafs) + __popc(leafs & ((1u << lo) - 1u));
            if (ci < s.node_count) {
                const uint32_t b = __ldg(s.node_brick + ci);
                if (b < s.brick_count) brick = b;
            }
        }
    }
    if (brick != NONE) {
        // traverseBrickAndReturnHit (SVOBrickDDA.cpp:187-225)
        const uint32_t bc = __ldg(s.coord + bounded(brick, s.brick_count, V_BRICK));
        const float bmn[3] = {float(int(bc & 0x3FFu) * 8), float(int((bc >> 10) & 0x3FFu) * 8),
                              float(int((bc >> 20) & 0x3FFu) * 8)};
        float tn[3], tf[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            // min / max of t0 = (bmn - lo) * inv, t1 = ((bmn + 8) - lo) * inv:
            // rounded multiplication by one factor is monotone, so the order
            // of t0 and t1 is the sign of inv (equal values are the same
            // number, a -0 among them included).  No operand is NaN.
            const float t0 = (bmn[i] - st.rb.lo[i]) * st.rb.inv[i];
            const float t1 = ((bmn[i] + 8.0f) - st.rb.lo[i]) * st.rb.inv[i];
            const bool pos = st.rb.inv[i] > 0.0f;
            tn[i] = pos ? t0 : t1;
            tf[i] = pos ? t1 : t0;
        }
        const float btmin = gmax(gmax(gmax(tn[0], tn[1]), tn[2]), st.tEntry);
        const float btmax = gmin(gmin(tf[0], tf[1]), tf[2]);
        if (brick_dda(s, brick, bmn, st.rb, btmin, btmax, h)) {
            h.brick = brick;
            h.node = st.parent;
            h.flags |= method << 4;
            h.scale = uint32_t(s.max_levels - 1);  // SVOBrickDDA.cpp:509
            h.iters = uint32_t(st.iter);
            h.run_iters = h.iters;
            h.run_grid_reads = h.grid_reads;
            h.run_dda_steps = h.dda_steps;
            return true;
        }
    }
    return false;
}

// executeAdvancePhase (:380-416) and, when the step leaves the parent,
// executePopPhase (:418-510).  Returns 1 when the ray is finished (it left
// the octree or the quantised position ends the traversal), else 0.
__device__ __forceinline__ bool advance_pop(const DevScene& s, CastState& st, const Corners& k, bool csx, bool csy,
                                            bool csz, uint32_t* stkN, float* stkT, int stride) {
    const Coef& c = st.c;
    const int minScale = s.min_scale;
    {
        float tca = k.tcc;
        if (tca == FLT_MAX_) tca = nmax3(csx ? k.tx : -FLT_MAX_, csy ? k.ty : -FLT_MAX_, csz ? k.tz : -FLT_MAX_);
        int step_mask = 0;
        if (csx && k.tx <= tca) { step_mask ^= 1; st.px -= st.scale_exp2; }
        if (csy && k.ty <= tca) { step_mask ^= 2; st.py -= st.scale_exp2; }
        if (csz && k.tz <= tca) { step_mask ^= 4; st.pz -= st.scale_exp2; }
        st.t_min = nmax(tca, 0.0f);
        st.idx ^= step_mask;
        if ((st.idx & step_mask) == 0) return false;
    }
    // POP: step mask recomputed at the new position (:672-681)
    int step_mask = 0;
    {
        const float ux = st.px * c.tx_coef - c.tx_bias;
        const float uy = st.py * c.ty_coef - c.ty_bias;
        const float uz = st.pz * c.tz_coef - c.tz_bias;
        const float ucc = nmin3((csx && fabsf(ux) < 1000.0f) ? ux : st.t_max,
                                (csy && fabsf(uy) < 1000.0f) ? uy : st.t_max,
                                (csz && fabsf(uz) < 1000.0f) ? uz : st.t_max);
        if (csx && ux <= ucc) step_mask ^= 1;
        if (csy && uy <= ucc) step_mask ^= 2;
        if (csz && uz <= ucc) step_mask ^= 4;
    }
    if (st.scale == ESVO_MAX_SCALE) {
        if (st.t_min > st.t_max || st.px < 1.0f || st.px >= 2.0f || st.py < 1.0f || st.py >= 2.0f || st.pz < 1.0f ||
            st.pz >= 2.0f) {
            cast_finish(st);
            return true;
        }
        st.fetched = false;
        return false;
    }
    // floatToInt: std::max(0, std::min(f, 1)), * 2^22, std::min(., 2^22-1),
    // std::max(0, .), truncate (SVOTraversal.cpp:439-442).  Every argument
    // here is max(0, .) of a finite value, so f >= +0 and both std::max
    // calls return their other operand.
    auto f2q = [](float f) -> uint32_t { return uint32_t(nmin(nmin(f, 1.0f) * 4194304.0f, 4194303.0f)); };
    uint32_t qx = f2q(nmax(0.0f, st.px - 1.0f));
    uint32_t qy = f2q(nmax(0.0f, st.py - 1.0f));
    uint32_t qz = f2q(nmax(0.0f, st.pz - 1.0f));
    uint32_t diff = 0;
    if (step_mask & 1) diff |= qx ^ f2q(nmax(0.0f, st.px + st.scale_exp2 - 1.0f));
    if (step_mask & 2) diff |= qy ^ f2q(nmax(0.0f, st.py + st.scale_exp2 - 1.0f));
    if (step_mask & 4) diff |= qz ^ f2q(nmax(0.0f, st.pz + st.scale_exp2 - 1.0f));
    if (diff == 0) { cast_finish(st); return true; }
    st.scale = 31 - __clz(diff);
    if (st.scale < minScale || st.scale > ESVO_MAX_SCALE) { cast_finish(st); return true; }
    st.scale_exp2 = __int_as_float((st.scale - ESVO_MAX_SCALE + 127) << 23);
    if ((st.pushed >> (st.scale - minScale)) & 1u) {
        const uint32_t kk = bounded(uint32_t(st.scale - minScale), uint32_t(s.max_levels), V_STACK);
        st.parent = stkN[kk * stride];
        st.t_max = stkT[kk * stride];
    } else {
        st.parent = 0u;
        st.t_max = st.t_root;
    }
    const uint32_t mask = ~((1u << (ESVO_MAX_SCALE - st.scale)) - 1u);
    qx &= mask; qy &= mask; qz &= mask;
    st.px = 1.0f + float(qx) * (1.0f / 4194304.0f);  // / 2^22, exact as a product
    st.py = 1.0f + float(qy) * (1.0f / 4194304.0f);
    st.pz = 1.0f + float(qz) * (1.0f / 4194304.0f);
    const int sh = ESVO_MAX_SCALE - st.scale - 1;
    if (sh < 0 || sh >= 32) st.idx = 0;
    else st.idx = int(((qx >> sh) & 1u) | (((qy >> sh) & 1u) << 1) | (((qz >> sh) & 1u) << 2));
    st.hh = 0.0f;
    st.fetched = false;
    return false;
}

// executePushPhase (:328-378) into the iteration's child (tx_center etc. of
// checkChildValidity): the parent goes on the stack when tc_max < h.
__device__ __forceinline__ void push_child(const DevScene& s, CastState& st, const Corners& k, int worldIdx,
                                           float tv_max, uint32_t* stkN, float* stkT, int stride) {
    const Coef& c = st.c;
    const int minScale = s.min_scale;
    const float half = st.scale_exp2 * 0.5f;
    const float tx_center = half * c.tx_coef + k.tx;
    const float ty_center = half * c.ty_coef + k.ty;
    const float tz_center = half * c.tz_coef + k.tz;
    const float tc_max = nmin3(k.tx, k.ty, k.tz);
    if (tc_max < st.hh) {
        const uint32_t kk = bounded(uint32_t(st.scale - minScale), uint32_t(s.max_levels), V_STACK);
        stkN[kk * stride] = st.parent;
        stkT[kk * stride] = st.t_max;
        st.pushed |= 1u << (st.scale - minScale);
    }
    st.hh = tc_max;
    const uint32_t nonLeafMask = ~(st.pMask >> 8) & st.pMask & 0xFFu;
    const uint32_t child_index = st.pChild + __popc(nonLeafMask & ((1u << worldIdx) - 1u));
    if (child_index < s.node_count) {
        st.parent = child_index;
        st.idx = 0;
        st.scale--;
        st.scale_exp2 = half;
        if (tx_center > st.t_min) { st.idx ^= 1; st.px += st.scale_exp2; }
        if (ty_center > st.t_min) { st.idx ^= 2; st.py += st.scale_exp2; }
        if (tz_center > st.t_min) { st.idx ^= 4; st.pz += st.scale_exp2; }
        st.t_max = tv_max;
        st.fetched = false;
    }
}

// Long cycles (Brent's method).  A state can also repeat after p > 2
// iterations; then the stack matters too, since a POP inside the cycle may
// read a slot that the cycle only writes after it.  At iterations 16, 32, 64,
// 128 and 256 the loop state, the pushed mask, the pushed stack slots and the
// counters are copied to the checkpoint `ck` (per-thread local memory, only
// touched there); a later state whose signature equals the checkpoint's is
// compared in full, stack included.  Equal means that every later iteration
// repeats the p = iter - iter(ck) iterations since the checkpoint, with the
// same counter increments, and that no hit or exit can come.  The whole
// cycles the 500-iteration cap leaves room for are then skipped (an even
// number when p is odd, so the short check's parity slots stay in step):
// iter and the counters advance by whole cycles and the loop goes on for the
// rest, fewer than 2p iterations, which ends at the cap with the reference's
// counters.  ck[12..14] keep the skipped iterations, grid reads and DDA steps
// so that the executed counts (run_*) can be restored (finish_skipped).
//   ck: [0..7] state words, [8] pushed mask, [9] iter, [10] grid reads,
//       [11] DDA steps, [12..14] skipped, [16 + 2j], [17 + 2j] stack slot j
__device__ __forceinline__ void long_cycle_checkpoint(const CastState& st, const uint32_t* cur, const uint32_t* stkN,
                                                      const float* stkT, int stride, uint32_t* ck) {
    const uint32_t pm = st.pushed & ~SKIPPED;
    for (int k = 0; k < 8; ++k) ck[k] = cur[k];
    ck[8] = pm;
    ck[9] = uint32_t(st.iter);
    ck[10] = st.h.grid_reads;
    ck[11] = st.h.dda_steps;
    for (uint32_t m = pm; m; m &= m - 1u) {
        const int j = __ffs(int(m)) - 1;
        ck[16 + 2 * j] = stkN[j * stride];
        ck[17 + 2 * j] = __float_as_uint(stkT[j * stride]);
    }
}

__device__ __forceinline__ bool long_cycle_equal(const CastState& st, const uint32_t* cur, const uint32_t* stkN,
                                                 const float* stkT, int stride, const uint32_t* ck) {
    bool eq = (st.pushed & ~SKIPPED) == ck[8];
    for (int k = 0; k < 8; ++k) eq = eq && cur[k] == ck[k];
    for (uint32_t m = ck[8]; eq && m; m &= m - 1u) {
        const int j = __ffs(int(m)) - 1;
        eq = stkN[j * stride] == ck[16 + 2 * j] && __float_as_uint(stkT[j * stride]) == ck[17 + 2 * j];
    }
    return eq;
}

__device__ __forceinline__ void long_cycle(CastState& st, uint32_t sig, const uint32_t* cur, const uint32_t* stkN,
                                           const float* stkT, int stride, uint32_t* ck) {
    Hit& h = st.h;
    if ((st.iter & (st.iter - 1)) == 0) {
        long_cycle_checkpoint(st, cur, stkN, stkT, stride, ck);
        st.ck_sig = sig;
    } else if (sig == st.ck_sig && long_cycle_equal(st, cur, stkN, stkT, stride, ck)) {
        const uint32_t p = uint32_t(st.iter) - ck[9];
        uint32_t m = uint32_t(MAX_ITER - st.iter) / p;
        if (p & 1u) m &= ~1u;
        if (m) {
            const uint32_t si = m * p, sg = m * (h.grid_reads - ck[10]), sd = m * (h.dda_steps - ck[11]);
            if (!(st.pushed & SKIPPED)) {
                ck[12] = ck[13] = ck[14] = 0u;
                st.pushed |= SKIPPED;
            }
            ck[12] += si;
            ck[13] += sg;
            ck[14] += sd;
            st.iter += int(si);
            h.grid_reads += sg;
            h.dda_steps += sd;
        }
    }
}

// After the ray has finished: run_* count what was executed, not the skipped cycles.
__device__ __forceinline__ void finish_skipped(CastState& st, const uint32_t* ck) {
    if (st.pushed & SKIPPED) {
        st.h.run_iters -= ck[12];
        st.h.run_grid_reads -= ck[13];
        st.h.run_dda_steps -= ck[14];
    }
}

// The end of an iteration: the cycle check (see above).  g0 / dd0: the grid
// reads and DDA steps counted when the iteration began.  True when a proven
// repeat ends the ray.
template <bool DEFER>
__device__ __forceinline__ bool cycle_check(CastState& st, uint32_t g0, uint32_t dd0, uint32_t* cyc, int stride,
                                            const uint32_t* stkN, const float* stkT, uint32_t* ck) {
    Hit& h = st.h;
    if (st.iter < CYCLE_START) return false;
    uint32_t cur[8];
    cur[0] = uint32_t(st.scale) | (uint32_t(st.idx) << 8) | (uint32_t(st.fetched) << 16);
    cur[1] = st.parent;
    cur[2] = __float_as_uint(st.px); cur[3] = __float_as_uint(st.py); cur[4] = __float_as_uint(st.pz);
    cur[5] = __float_as_uint(st.t_min); cur[6] = __float_as_uint(st.t_max); cur[7] = __float_as_uint(st.hh);
    const uint32_t dg = h.grid_reads - g0, ddd = h.dda_steps - dd0;
    // signature: the words' sum (a repeat always has an equal sum)
    const uint32_t sig = ((cur[0] + cur[1] + cur[2]) + (cur[3] + cur[4] + cur[5])) + (cur[6] + cur[7]);
    int period = 0;  // 1 or 2 once state(iter) == state(iter - period) is proven
    if constexpr (!DEFER) {
        uint32_t* back2 = cyc + ((st.iter & 1) * 8) * stride;
        const uint32_t* back1 = cyc + (((st.iter & 1) ^ 1) * 8) * stride;
        bool eq1 = st.iter >= CYCLE_START + 1 && st.sig1 == sig;
        bool eq2 = st.iter >= CYCLE_START + 2 && st.sig2 == sig;
        if (eq1 || eq2) {
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                eq1 = eq1 && (cur[k] == back1[k * stride]);
                eq2 = eq2 && (cur[k] == back2[k * stride]);
            }
        }
        period = eq1 ? 1 : (eq2 ? 2 : 0);
        if (!period) {
#pragma unroll
            for (int k = 0; k < 8; ++k) back2[k * stride] = cur[k];
        }
    } else {
        if (st.cand_p && st.iter == st.cand_at) {
            bool eq = true;
#pragma unroll
            for (int k = 0; k < 8; ++k) eq = eq && (cur[k] == cyc[k * stride]);
            if (eq) period = st.cand_p;
            st.cand_p = 0;
        }
        if (!period && !st.cand_p) {
            const int p = (st.iter >= CYCLE_START + 1 && sig == st.sig1)
                              ? 1
                              : ((st.iter >= CYCLE_START + 2 && sig == st.sig2) ? 2 : 0);
            if (p) {
#pragma unroll
                for (int k = 0; k < 8; ++k) cyc[k * stride] = cur[k];
                st.cand_p = p;
                st.cand_at = st.iter + p;
            }
        }
    }
    if (period) {  // the rest of the 500 iterations repeat the cycle: the capped miss
        const uint32_t rem = uint32_t(MAX_ITER - st.iter);
        h.run_iters = uint32_t(st.iter);
        h.run_grid_reads = h.grid_reads;
        h.run_dda_steps = h.dda_steps;
        if (period == 1) {
            h.grid_reads += rem * dg;
            h.dda_steps += rem * ddd;
        } else {
            h.grid_reads += ((rem + 1) / 2) * st.d1g + (rem / 2) * dg;
            h.dda_steps += ((rem + 1) / 2) * st.d1d + (rem / 2) * ddd;
        }
        h.iters = uint32_t(MAX_ITER);
        h.flags |= F_ITER_CAP;
        return true;
    }
    if (st.iter >= LONG_FIRST) long_cycle(st, sig, cur, stkN, stkT, stride, ck);
    st.sig2 = st.sig1;
    st.sig1 = sig;
    st.d1g = dg;
    st.d1d = ddd;
    return false;
}

// One iteration, its loop condition first.  Returns true when the ray is
// finished (hit, exit, cap).  MERGE: how the branches after the child test are
// laid out (same operations and results either way).
template <bool LOD = false, bool DEFER = false, bool MERGE = false>
__device__ __forceinline__ bool cast_step(const DevScene& s, CastState& st, uint32_t* stkN, float* stkT,
                                          uint32_t* cyc, int stride, uint32_t* ck,
                                          LodCone lod = LodCone{0.0f, 0.0f}) {
    Hit& h = st.h;
    const Coef& c = st.c;
    const int minScale = s.min_scale;
    if (!(st.scale >= minScale && st.scale <= ESVO_MAX_SCALE && st.iter < MAX_ITER)) {
        cast_finish(st);
        return true;
    }
    const bool csx = fabsf(st.dx) >= 1e-5f, csy = fabsf(st.dy) >= 1e-5f, csz = fabsf(st.dz) >= 1e-5f;
    ++st.iter;
    const uint32_t g0 = h.grid_reads, dd0 = h.dda_steps;
    // fetchChildDescriptor (:282-293)
    if (!st.fetched) {
        const uint2 nd = __ldg(s.nodes + bounded(st.parent, s.node_count, V_NODE));
        st.pChild = nd.x;
        st.pMask = nd.y & 0xFFFFu;
        // a descriptor reads as fetched unless it is all zero (child pointer 0,
        // no valid child, all eight leaf bits clear); mirroring keeps a mask's
        // zeroness
        st.fetched = ((st.pMask & 0xFFu) | (~st.pMask & 0xFF00u) | st.pChild) != 0u;
    }
    const Corners k = corners_of(st, csx, csy, csz);
    // checkChildValidity (:295-326)
    const int worldIdx = st.idx ^ (~c.octant_mask & 7);
    const bool child_valid = (st.pMask >> worldIdx) & 1u;
    bool isLeaf = (st.pMask >> (worldIdx + 8)) & 1u;
    if (st.scale - minScale == s.brick_user_scale && child_valid) isLeaf = true;
    float tv_max = 0.0f;
    // !(t_min > t_max) && t_min <= min(t_max, tc_max): the first test follows
    // from the second, the loop's t values being NaN-free
    const bool in_range = child_valid && st.t_min <= (tv_max = nmin(st.t_max, k.tcc));
    if (in_range) {
        if constexpr (LOD) {
            // worldDistance = tRayStart + t_min * |worldSize| (:627);
            // esvoScaleToWorldSize = 2^(scale - 23) * worldSize.x (SVOLOD.h:189-195),
            // an exact power of two for scale in [0, 22];
            // shouldTerminate: distance * rayDirSize + rayOrigSize >= size (SVOLOD.h:129-146).
            const float wd = st.tRayStart + st.t_min * s.wrl;
            const float vs = __int_as_float((st.scale - ESVO_MAX_SCALE - 1 + 127) << 23) * s.wsize[0];
            if (wd * lod.dir + lod.orig >= vs) {
                // The LOD hit (:639-649): tMin = distance, normal (0,1,0), no entity.
                h.t = wd;
                h.node = st.parent;
                h.flags = F_HIT | (1u << 1);
                h.scale = uint32_t(st.scale - minScale);  // esvoToUserScale
                cast_finish(st);
                return true;
            }
        }
    }
    if constexpr (MERGE) {
        // A leaf child in range: the leaf stage; when its brick is not hit the
        // iteration continues with ADVANCE from tv_max, like a child out of
        // range, and both run the one ADVANCE below (lanes of a warp that took
        // either way stay converged there: incoherent rays).
        if (in_range && isLeaf) {
            if (leaf_stage(s, st, csx, csy, csz)) return true;
            st.t_min = tv_max;
        }
        if (in_range && !isLeaf) push_child(s, st, k, worldIdx, tv_max, stkN, stkT, stride);
        else if (advance_pop(s, st, k, csx, csy, csz, stkN, stkT, stride)) return true;
    } else {
        // The same iteration as the reference writes its branches (coherent
        // rays, whose warps take one way at a time).
        if (in_range) {
            if (isLeaf) {
                if (leaf_stage(s, st, csx, csy, csz)) return true;
                st.t_min = tv_max;
                if (advance_pop(s, st, k, csx, csy, csz, stkN, stkT, stride)) return true;
            } else {
                push_child(s, st, k, worldIdx, tv_max, stkN, stkT, stride);
            }
        } else if (advance_pop(s, st, k, csx, csy, csz, stkN, stkT, stride)) {
            return true;
        }
    }
    return cycle_check<DEFER>(st, g0, dd0, cyc, stride, stkN, stkT, ck);
}

// castRayImpl (SVOTraversal.cpp:516-691): setup, then the loop.  LOD = false
// is castRay, LOD = true castRayWithLOD with an enabled `lod`.
template <bool LOD = false, bool DEFER = false>
__device__ __forceinline__ void cast_ray(const DevScene& s, float ox, float oy, float oz, float ddx, float ddy,
                                         float ddz, float tMinArg, float tMaxArg, uint32_t* stkN, float* stkT,
                                         uint32_t* cyc, int stride, Hit& h, LodCone lod = LodCone{0.0f, 0.0f}) {
    CastState st;
    uint32_t ck[CK_WORDS];
    if (!cast_init(s, ox, oy, oz, ddx, ddy, ddz, tMinArg, tMaxArg, stkN, stkT, stride, st)) {
        while (!cast_step<LOD, DEFER>(s, st, stkN, stkT, cyc, stride, ck, lod)) {
        }
        finish_skipped(st, ck);
    }
    h = st.h;
}

// cast_ray that gives up once `budget` iterations have run without ending the
// ray: false then, and h is not written.  The cast is deterministic, so the
// caller can cast the ray again from the start for its result.
template <bool LOD = false, bool DEFER = false, bool MERGE = false>
__device__ __forceinline__ bool cast_ray_budget(const DevScene& s, float ox, float oy, float oz, float ddx, float ddy,
                                                float ddz, float tMinArg, float tMaxArg, uint32_t* stkN, float* stkT,
                                                uint32_t* cyc, int stride, int budget, Hit& h) {
    CastState st;
    uint32_t ck[CK_WORDS];
    if (!cast_init(s, ox, oy, oz, ddx, ddy, ddz, tMinArg, tMaxArg, stkN, stkT, stride, st)) {
        // every cast_step that returns false has counted one iteration in st.iter
        while (!cast_step<LOD, DEFER, MERGE>(s, st, stkN, stkT, cyc, stride, ck)) {
            if (st.iter >= budget) return false;
        }
        finish_skipped(st, ck);
    }
    h = st.h;
    return true;
}

// DXT1 texel of the hit voxel: decodeColorHead (DXT1Compressor.cpp:14-36)
// and the compressed shader's addressing (VoxelRayMarch_Compressed.comp:142-158).
__device__ __forceinline__ void dxt_texel(const uint2* dxt, uint32_t brick, uint32_t voxel, float& r, float& g,
                                          float& b) {
    const uint2 blk = __ldg(dxt + size_t(brick) * 32 + (voxel >> 4));
    const uint32_t head = blk.x;
    const uint32_t sel = (blk.y >> ((voxel & 15u) * 2u)) & 3u;
    const float scale = 1.0f / 4294967296.0f;
    const float r0x = float(head << 16) * scale, r0y = float(head << 21) * scale, r0z = float(head << 27) * scale;
    const float r1x = float(head) * scale, r1y = float(head << 5) * scale, r1z = float(head << 11) * scale;
    // The shader's four cases as one blend r0 * w0 + r1 * w1, (w0, w1) = (1, 0), (0, 1),
    // (2/3, 1/3), (1/3, 2/3) for selectors 0..3: the same roundings (the endpoints are finite
    // and non-negative, so x * 1 = x and x * 0 + y = y exactly), without a branch per selector
    // (neighbouring voxels of a warp have different selectors).
    const float w0 = sel == 0u ? 1.0f : (sel == 1u ? 0.0f : (sel == 2u ? 2.0f / 3.0f : 1.0f / 3.0f));
    const float w1 = sel == 0u ? 0.0f : (sel == 1u ? 1.0f : (sel == 2u ? 1.0f / 3.0f : 2.0f / 3.0f));
    r = r0x * w0 + r1x * w1;
    g = r0y * w0 + r1y * w1;
    b = r0z * w0 + r1z * w1;
}

// getCompressedVoxelNormal (VoxelRayMarch_Compressed.comp:160-165):
// normalize(decodeDXTNormal) of the voxel's texel (Compression.glsl:158-177).
__device__ __forceinline__ void dxt_normal(const DevScene& s, uint32_t brick, uint32_t voxel, float& x, float& y,
                                           float& z) {
    const uint4 q = __ldg(s.nrm + size_t(bounded(brick, s.brick_count, V_BRICK)) * 32 +
                          (bounded(voxel, 512u, V_VOXEL) >> 4));
    const dxtn::F3 n = dxtn::unit(dxtn::decode(uint64_t(q.x) | (uint64_t(q.y) << 32),
                                               uint64_t(q.z) | (uint64_t(q.w) << 32), voxel & 15u));
    x = n.x; y = n.y; z = n.z;
}

__device__ __forceinline__ void store_hit(vx_hit* hits, uint32_t i, const Hit& h) {
    uint4 v;
    v.x = __float_as_uint(h.t);
    v.y = h.brick;
    v.z = h.node;
    v.w = (h.voxel & 0xFFFFu) | ((h.flags & 0xFFu) << 16) | (h.scale << 24);
    reinterpret_cast<uint4*>(hits)[i] = v;
}

// Colour of the hit voxel (the RGBA8 or material word, or the decoded DXT1
// texel); 0 on a miss and on an LOD hit (no voxel).
__device__ __forceinline__ void store_color(const DevScene& s, void* color, uint32_t i, const Hit& h) {
    const bool hit = (h.flags & F_HIT) && h.brick != NONE;
    if (s.color_kind == VX_COLOR_RGBA8 || s.color_kind == VX_COLOR_MATERIAL) {
        reinterpret_cast<uint32_t*>(color)[i] =
            hit ? __ldg(s.rgba + size_t(bounded(h.brick, s.brick_count, V_BRICK)) * 512 +
                        bounded(h.voxel, 512u, V_VOXEL))
                : 0u;
    } else if (s.color_kind == VX_COLOR_DXT1) {
        float r = 0.0f, g = 0.0f, b = 0.0f;
        if (hit) dxt_texel(s.dxt, bounded(h.brick, s.brick_count, V_BRICK), bounded(h.voxel, 512u, V_VOXEL), r, g, b);
        float* c = reinterpret_cast<float*>(color) + size_t(i) * 3;
        c[0] = r; c[1] = g; c[2] = b;
    }
}

}  // namespace
// Host reader of this translation unit's violation word (read and clear).
#if VX_CHECKED
#define VX_VIOLATION_READER(fn)                                              \
    uint32_t fn() {                                                          \
        unsigned int v = 0u, z = 0u;                                         \
        if (cudaMemcpyFromSymbol(&v, vx_violation, sizeof(v)) != cudaSuccess) \
            return 0x80000000u;                                              \
        cudaMemcpyToSymbol(vx_violation, &z, sizeof(z));                     \
        return v;                                                            \
    }
#else
#define VX_VIOLATION_READER(fn) \
    uint32_t fn() { return 0u; }
#endif

}  // namespace vx
