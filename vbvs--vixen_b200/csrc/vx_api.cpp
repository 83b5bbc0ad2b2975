// vx_api.cpp - host side of the C ABI (include/vx.h): validation, the scene's
// device allocation, error reporting and launches.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "vx_internal.h"
#include "vx_raygen.h"

namespace vx {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

const char* last_error_c_str() { return g_last_error.c_str(); }

int cuda_fail(cudaError_t e, const std::string& what) {
    return fail(VX_ECUDA, what + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

CameraDev camera_from_pc(const vx_camera_pc& pc) {
    CameraDev c{};
    for (int i = 0; i < 3; ++i) {
        c.pos[i] = pc.camera_pos[i];
        c.dir[i] = pc.camera_dir[i];
        c.up[i] = pc.camera_up[i];
        c.right[i] = pc.camera_right[i];
    }
    c.aspect = pc.aspect;
    // tan(radians(fov * 0.5)) (RayGeneration.glsl:62), once, in binary32.
    const float half = pc.fov * 0.5f;
    const float rad = half * 0.01745329251994329577f;
    c.tan_half_fov = std::tan(rad);
    return c;
}

}  // namespace vx

// Copy / cast pipeline of the host-buffer casts: smallest chunk (rays) and
// most chunks per call.
#ifndef VX_PIPE_MIN_CHUNK
#define VX_PIPE_MIN_CHUNK 524288u
#endif
#ifndef VX_PIPE_MAX_CHUNKS
#define VX_PIPE_MAX_CHUNKS 16u
#endif
#ifndef VX_PIPE_CAST_STREAMS
#define VX_PIPE_CAST_STREAMS 4
#endif

struct vx_scene {
    int device = 0;
    vx_octree_config cfg{};
    void* pool = nullptr;  // single device allocation, 256-byte aligned slices
    uint64_t pool_bytes = 0;
    vx::DevScene dev{};
    // staging buffer for vx_cast_rays_host, grown on demand, and the streams
    // and events of its copy / cast pipeline (created on first use)
    std::mutex stage_mu;
    void* stage = nullptr;
    uint64_t stage_bytes = 0;
    cudaStream_t pipe[2 + VX_PIPE_CAST_STREAMS] = {};  // copies in, copies out, casts
    cudaEvent_t pipe_start = nullptr;
    cudaEvent_t pipe_in[VX_PIPE_MAX_CHUNKS] = {}, pipe_cast[VX_PIPE_MAX_CHUNKS] = {};
    // scratch of vx_cast_shadow_rays (compacted shadow rays and their slots), grown on demand
    void* shadow = nullptr;
    uint64_t shadow_bytes = 0;
};

namespace vx {
const DevScene& scene_dev(const vx_scene* s) { return s->dev; }
int scene_device(const vx_scene* s) { return s->device; }

namespace {
uint64_t align256_(uint64_t x) { return (x + 255) & ~uint64_t(255); }
}  // namespace

// One cudaMalloc with 256-byte aligned slices, like the reference's single
// VkDeviceMemory with aligned sub-buffers (VoxelSceneCacher.cpp:736-869).
int scene_alloc(const vx_octree_config& c, uint32_t node_count, uint32_t brick_count, int32_t color_kind,
                bool normals, vx_scene** out, ScenePool* p) {
    *out = nullptr;
    const uint64_t bpa = uint64_t(c.bricks_per_axis);
    ScenePool q{};
    q.sz_nodes = uint64_t(node_count) * sizeof(vx_node);
    q.sz_nb = uint64_t(node_count) * 4;
    q.sz_grid = bpa * bpa * bpa * 4;
    q.sz_coord = uint64_t(brick_count) * 4;
    q.sz_occ = uint64_t(brick_count) * 64;
    if (color_kind == VX_COLOR_RGBA8 || color_kind == VX_COLOR_MATERIAL) q.sz_color = uint64_t(brick_count) * 512 * 4;
    if (color_kind == VX_COLOR_DXT1) q.sz_color = uint64_t(brick_count) * 32 * 8;
    q.sz_nrm = normals ? uint64_t(brick_count) * 32 * 16 : 0;
    const uint64_t o_nodes = 0;
    const uint64_t o_nb = o_nodes + align256_(q.sz_nodes);
    const uint64_t o_grid = o_nb + align256_(q.sz_nb);
    const uint64_t o_coord = o_grid + align256_(q.sz_grid);
    const uint64_t o_occ = o_coord + align256_(q.sz_coord);
    const uint64_t o_color = o_occ + align256_(q.sz_occ);
    const uint64_t o_nrm = o_color + align256_(q.sz_color);
    const uint64_t total = o_nrm + align256_(q.sz_nrm) + 256;
    auto* s = new (std::nothrow) vx_scene();
    if (!s) return fail(VX_ENOMEM, "scene: out of host memory");
    cudaError_t e = cudaGetDevice(&s->device);
    if (e != cudaSuccess) { delete s; return cuda_fail(e, "scene: cudaGetDevice"); }
    e = cudaMalloc(&s->pool, total);
    if (e != cudaSuccess) { delete s; return cuda_fail(e, "scene: cudaMalloc"); }
    s->pool_bytes = total;
    char* base = static_cast<char*>(s->pool);
    q.nodes = base + o_nodes;
    q.node_brick = base + o_nb;
    q.grid = base + o_grid;
    q.coord = base + o_coord;
    q.occ = base + o_occ;
    q.color = q.sz_color ? base + o_color : nullptr;
    q.nrm = q.sz_nrm ? base + o_nrm : nullptr;
    DevScene& ds = s->dev;
    for (int i = 0; i < 3; ++i) {
        ds.wmin[i] = c.world_min[i];
        ds.wmax[i] = c.world_max[i];
        ds.wsize[i] = c.world_max[i] - c.world_min[i];
        ds.wsm[i] = ds.wsize[i] - 0.001f;
        ds.qwm[i] = int32_t(std::floor(c.world_min[i]));
    }
    for (int i = 0; i < 3; ++i) {
        int e = 0;
        const float m = std::frexp(ds.wsize[i], &e);  // wsize = m * 2^e, m in [0.5, 1)
        ds.wsinv[i] = (m == 0.5f && e - 1 > -126 && e - 1 < 126) ? std::ldexp(1.0f, 1 - e) : 0.0f;
    }
    // glm::length: sqrt of the left-to-right dot product
    ds.wrl = std::sqrt((ds.wsize[0] * ds.wsize[0] + ds.wsize[1] * ds.wsize[1]) + ds.wsize[2] * ds.wsize[2]);
    ds.max_levels = c.max_levels;
    ds.min_scale = 22 - c.max_levels + 1;
    ds.brick_user_scale = c.max_levels - c.brick_depth;
    ds.bpa = c.bricks_per_axis;
    ds.node_count = node_count;
    ds.brick_count = brick_count;
    ds.nodes = reinterpret_cast<const uint2*>(q.nodes);
    ds.node_brick = reinterpret_cast<const uint32_t*>(q.node_brick);
    ds.grid = reinterpret_cast<const uint32_t*>(q.grid);
    ds.coord = reinterpret_cast<const uint32_t*>(q.coord);
    ds.occ = reinterpret_cast<const uint4*>(q.occ);
    ds.color_kind = color_kind;
    ds.rgba = (color_kind == VX_COLOR_RGBA8 || color_kind == VX_COLOR_MATERIAL) ? reinterpret_cast<const uint32_t*>(q.color)
                                                                                : nullptr;
    ds.dxt = color_kind == VX_COLOR_DXT1 ? reinterpret_cast<const uint2*>(q.color) : nullptr;
    ds.nrm = reinterpret_cast<const uint4*>(q.nrm);
    s->cfg = c;
    *p = q;
    *out = s;
    return VX_OK;
}

}  // namespace vx

namespace {

using vx::fail;

uint64_t align256(uint64_t x) { return (x + 255) & ~uint64_t(255); }

// Host-side checks that make every device read in bounds: grid entries and
// node brick fields are brick indices or 0xFFFFFFFF, coordinates lie in the
// grid.  Child pointers are not rejected: the traversal bounds-checks them
// exactly as executePushPhase does (SVOTraversal.cpp:352-354).
int validate(const vx_scene_desc* d) {
    const vx_octree_config& c = d->config;
    if (c.brick_depth != 3) return fail(VX_EINVAL, "vx_scene_create: brick_depth must be 3 (8^3 bricks)");
    if (c.max_levels < 1 || c.max_levels > 23) return fail(VX_EINVAL, "vx_scene_create: max_levels must be in [1, 23]");
    if (c.bricks_per_axis < 1 || c.bricks_per_axis > 1024)
        return fail(VX_EINVAL, "vx_scene_create: bricks_per_axis must be in [1, 1024]");
    for (int i = 0; i < 3; ++i)
        if (!std::isfinite(c.world_min[i]) || !std::isfinite(c.world_max[i]) || !(c.world_max[i] > c.world_min[i]))
            return fail(VX_EINVAL, "vx_scene_create: world bounds must be finite with max > min");
    const float wsx = c.world_max[0] - c.world_min[0];
    const int vpa = (wsx < 2147483648.0f) ? int(wsx) : -1;
    if (vpa < 0 || (vpa + 7) / 8 != c.bricks_per_axis)
        return fail(VX_EINVAL, "vx_scene_create: bricks_per_axis must be ceil(int(world_max.x - world_min.x) / 8)");
    if (d->node_count && (!d->nodes || !d->node_brick)) return fail(VX_EINVAL, "vx_scene_create: nodes missing");
    if (!d->grid_lookup) return fail(VX_EINVAL, "vx_scene_create: grid_lookup missing");
    if (d->brick_count && (!d->brick_coord || !d->brick_occ))
        return fail(VX_EINVAL, "vx_scene_create: brick buffers missing");
    if (d->color_kind != VX_COLOR_NONE && d->color_kind != VX_COLOR_RGBA8 && d->color_kind != VX_COLOR_DXT1 &&
        d->color_kind != VX_COLOR_MATERIAL)
        return fail(VX_EINVAL, "vx_scene_create: unknown color_kind");
    if (d->color_kind != VX_COLOR_NONE && d->brick_count && !d->brick_color)
        return fail(VX_EINVAL, "vx_scene_create: brick_color missing");
    const uint64_t slots = uint64_t(c.bricks_per_axis) * c.bricks_per_axis * c.bricks_per_axis;
    for (uint64_t i = 0; i < slots; ++i)
        if (d->grid_lookup[i] != 0xFFFFFFFFu && d->grid_lookup[i] >= d->brick_count)
            return fail(VX_EINVAL, "vx_scene_create: grid_lookup[" + std::to_string(i) + "] is not a brick index");
    const uint32_t bpa = uint32_t(c.bricks_per_axis);
    for (uint32_t b = 0; b < d->brick_count; ++b) {
        const uint32_t v = d->brick_coord[b];
        if ((v & 0x3FF) >= bpa || ((v >> 10) & 0x3FF) >= bpa || ((v >> 20) & 0x3FF) >= bpa || (v >> 30))
            return fail(VX_EINVAL, "vx_scene_create: brick_coord[" + std::to_string(b) + "] outside the grid");
    }
    return VX_OK;
}

}  // namespace

extern "C" {

int32_t vx_abi_version(void) { return VX_ABI_VERSION; }

const char* vx_last_error_string(void) { return vx::last_error_c_str(); }

int vx_scene_create(const vx_scene_desc* d, vx_scene** out) {
    if (!d || !out) return fail(VX_EINVAL, "vx_scene_create: null argument");
    *out = nullptr;
    if (int r = validate(d)) return r;
    vx::ScenePool p;
    vx_scene* s = nullptr;
    if (int r = vx::scene_alloc(d->config, d->node_count, d->brick_count, d->color_kind, d->brick_normal != nullptr,
                                &s, &p))
        return r;
    struct Copy { void* dst; const void* src; uint64_t n; };
    const Copy copies[] = {{p.nodes, d->nodes, p.sz_nodes}, {p.node_brick, d->node_brick, p.sz_nb},
                           {p.grid, d->grid_lookup, p.sz_grid}, {p.coord, d->brick_coord, p.sz_coord},
                           {p.occ, d->brick_occ, p.sz_occ}, {p.color, d->brick_color, p.sz_color},
                           {p.nrm, d->brick_normal, p.sz_nrm}};
    for (const Copy& cp : copies) {
        if (!cp.n) continue;
        cudaError_t e = cudaMemcpy(cp.dst, cp.src, cp.n, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            vx_scene_destroy(s);
            return vx::cuda_fail(e, "vx_scene_create: cudaMemcpy");
        }
    }
    *out = s;
    return VX_OK;
}

int vx_scene_destroy(vx_scene* s) {
    if (!s) return VX_OK;
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev != s->device) cudaSetDevice(s->device);
    for (cudaStream_t& p : s->pipe)
        if (p) cudaStreamDestroy(p);
    if (s->pipe_start) cudaEventDestroy(s->pipe_start);
    for (uint32_t i = 0; i < VX_PIPE_MAX_CHUNKS; ++i) {
        if (s->pipe_in[i]) cudaEventDestroy(s->pipe_in[i]);
        if (s->pipe_cast[i]) cudaEventDestroy(s->pipe_cast[i]);
    }
    // Every buffer is freed whatever the others' outcome; the first error is reported.
    const cudaError_t e1 = cudaFree(s->pool);
    const cudaError_t e2 = s->stage ? cudaFree(s->stage) : cudaSuccess;
    const cudaError_t e3 = s->shadow ? cudaFree(s->shadow) : cudaSuccess;
    if (dev >= 0 && dev != s->device) cudaSetDevice(dev);
    delete s;
    for (cudaError_t e : {e1, e2, e3})
        if (e != cudaSuccess) return vx::cuda_fail(e, "vx_scene_destroy: cudaFree");
    return VX_OK;
}

int vx_bounds_checks(int32_t* enabled, uint32_t* violations) {
#ifndef VX_CHECKED
#define VX_CHECKED 0
#endif
    if (enabled) *enabled = VX_CHECKED;
    if (violations) {
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) return vx::cuda_fail(e, "vx_bounds_checks: synchronize");
        *violations = vx::violations_kernels() | vx::violations_batch() | vx::violations_diff() |
                      vx::violations_payload();
    }
    return VX_OK;
}

int vx_scene_info_get(const vx_scene* s, vx_scene_info* out) {
    if (!s || !out) return fail(VX_EINVAL, "vx_scene_info_get: null argument");
    vx_scene_info i{};
    i.config = s->cfg;
    i.node_count = s->dev.node_count;
    i.brick_count = s->dev.brick_count;
    i.color_kind = s->dev.color_kind;
    i.has_normals = s->dev.nrm != nullptr;
    *out = i;
    return VX_OK;
}

int vx_scene_download(const vx_scene* s, uint32_t* nodes, uint32_t* node_brick, uint32_t* grid_lookup,
                      uint32_t* brick_coord, uint32_t* brick_occ, void* brick_color, uint64_t* brick_normal) {
    if (!s) return fail(VX_EINVAL, "vx_scene_download: null scene");
    const vx::DevScene& d = s->dev;
    const uint64_t bpa = uint64_t(d.bpa), B = d.brick_count;
    const uint64_t colw = (d.color_kind == VX_COLOR_RGBA8 || d.color_kind == VX_COLOR_MATERIAL) ? 512 * 4
                          : d.color_kind == VX_COLOR_DXT1                                   ? 32 * 8
                                                                                            : 0;
    const void* color_src = d.rgba ? static_cast<const void*>(d.rgba) : static_cast<const void*>(d.dxt);
    struct Copy { void* dst; const void* src; uint64_t n; };
    const Copy copies[] = {{nodes, d.nodes, uint64_t(d.node_count) * 8}, {node_brick, d.node_brick, uint64_t(d.node_count) * 4},
                           {grid_lookup, d.grid, bpa * bpa * bpa * 4}, {brick_coord, d.coord, B * 4},
                           {brick_occ, d.occ, B * 64}, {brick_color, color_src, B * colw},
                           {brick_normal, d.nrm, d.nrm ? B * 512 : 0}};
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev != s->device) cudaSetDevice(s->device);
    cudaError_t e = cudaSuccess;
    for (const Copy& c : copies)
        if (c.dst && c.n && e == cudaSuccess) e = cudaMemcpy(c.dst, c.src, c.n, cudaMemcpyDeviceToHost);
    if (dev >= 0 && dev != s->device) cudaSetDevice(dev);
    if (e != cudaSuccess) return vx::cuda_fail(e, "vx_scene_download");
    return VX_OK;
}

int vx_scene_device_bytes(const vx_scene* s, uint64_t* out) {
    if (!s || !out) return fail(VX_EINVAL, "vx_scene_device_bytes: null argument");
    *out = s->pool_bytes;
    return VX_OK;
}

namespace {

bool lod_ok(const vx_lod_params* lod) {
    return !lod || (std::isfinite(lod->ray_orig_size) && std::isfinite(lod->ray_dir_size));
}

int cast_rays_dev(const char* what, const vx_scene* s, const vx_ray* rays, uint32_t n, float tmin, float tmax,
                  const vx_lod_params* lod, vx_hit* hits, void* color, vx_ray_counters* counters, void* stream) {
    if (!s || (n && (!rays || !hits))) return fail(VX_EINVAL, std::string(what) + ": null argument");
    if (std::isnan(tmin) || std::isnan(tmax)) return fail(VX_EINVAL, std::string(what) + ": t_min / t_max is NaN");
    if (!lod_ok(lod)) return fail(VX_EINVAL, std::string(what) + ": LOD sizes must be finite");
    if (reinterpret_cast<uintptr_t>(rays) % 8 || reinterpret_cast<uintptr_t>(hits) % 16 ||
        reinterpret_cast<uintptr_t>(color) % 4 || reinterpret_cast<uintptr_t>(counters) % 16)
        return fail(VX_EINVAL,
                    std::string(what) + ": rays need 8-byte, hits and counters 16-byte, colour 4-byte alignment");
    int r = vx::launch_cast(s->dev, rays, n, tmin, tmax, hits, color, counters, stream, lod);
    if (r != 0) return vx::cuda_fail(cudaError_t(r), std::string(what) + ": launch");
    return VX_OK;
}

int cast_rays_host(const char* what, const vx_scene* cs, const vx_ray* rays_host, uint32_t n, float tmin,
                   float tmax, const vx_lod_params* lod, vx_hit* hits_host, void* color_host, void* stream) {
    const std::string w(what);
    if (!cs || (n && (!rays_host || !hits_host))) return fail(VX_EINVAL, w + ": null argument");
    if (std::isnan(tmin) || std::isnan(tmax)) return fail(VX_EINVAL, w + ": t_min / t_max is NaN");
    if (!lod_ok(lod)) return fail(VX_EINVAL, w + ": LOD sizes must be finite");
    if (n == 0) return VX_OK;
    vx_scene* s = const_cast<vx_scene*>(cs);
    std::lock_guard<std::mutex> lk(s->stage_mu);
    const uint64_t colw = s->dev.color_kind == VX_COLOR_DXT1 ? 12 : 4;
    const uint64_t sz_r = align256(uint64_t(n) * sizeof(vx_ray));
    const uint64_t sz_h = align256(uint64_t(n) * sizeof(vx_hit));
    const uint64_t sz_c = color_host && s->dev.color_kind != VX_COLOR_NONE ? align256(uint64_t(n) * colw) : 0;
    const uint64_t need = sz_r + sz_h + sz_c;
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev != s->device) return fail(VX_EINVAL, w + ": the scene belongs to another device");
    if (need > s->stage_bytes) {
        if (s->stage) cudaFree(s->stage);
        s->stage = nullptr;
        s->stage_bytes = 0;
        cudaError_t e = cudaMalloc(&s->stage, need);
        if (e != cudaSuccess) return vx::cuda_fail(e, w + ": cudaMalloc");
        s->stage_bytes = need;
    }
    char* base = static_cast<char*>(s->stage);
    vx_ray* dr = reinterpret_cast<vx_ray*>(base);
    vx_hit* dh = reinterpret_cast<vx_hit*>(base + sz_r);
    char* dc = sz_c ? base + sz_r + sz_h : nullptr;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!s->pipe_start) {
        cudaError_t e = cudaEventCreateWithFlags(&s->pipe_start, cudaEventDisableTiming);
        for (int i = 0; i < 2 + VX_PIPE_CAST_STREAMS && e == cudaSuccess; ++i)
            e = cudaStreamCreateWithFlags(&s->pipe[i], cudaStreamNonBlocking);
        for (uint32_t i = 0; i < VX_PIPE_MAX_CHUNKS && e == cudaSuccess; ++i) {
            e = cudaEventCreateWithFlags(&s->pipe_in[i], cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->pipe_cast[i], cudaEventDisableTiming);
        }
        if (e != cudaSuccess) return vx::cuda_fail(e, w + ": pipeline streams");
    }
    // The rays go in, are cast and come back out in chunks: one stream streams
    // the chunks in, each chunk is cast on one of VX_PIPE_CAST_STREAMS streams
    // once it has arrived (so the long last rays of one chunk overlap the next
    // chunk's cast), and one stream returns each chunk once it is cast.  The
    // two copy directions and the casts overlap (with pinned host buffers), and
    // no copy-in waits behind a cast.  Everything starts after the work
    // already queued on the caller's stream.
    const uint32_t min_chunk = VX_PIPE_MIN_CHUNK;
    const uint32_t chunks = n >= 2 * min_chunk ? std::min<uint32_t>(VX_PIPE_MAX_CHUNKS, n / min_chunk) : 1;
    cudaStream_t s_in = s->pipe[0], s_out = s->pipe[1];
    cudaError_t e = cudaEventRecord(s->pipe_start, st);
    for (int i = 0; i < 2 + VX_PIPE_CAST_STREAMS && e == cudaSuccess; ++i)
        e = cudaStreamWaitEvent(s->pipe[i], s->pipe_start, 0);
    if (e != cudaSuccess) return vx::cuda_fail(e, w + ": order");
    const char* rh = reinterpret_cast<const char*>(rays_host);
    char* hh = reinterpret_cast<char*>(hits_host);
    char* ch = static_cast<char*>(color_host);
    for (uint32_t c = 0; c < chunks; ++c) {
        const uint64_t a = uint64_t(n) * c / chunks, b = uint64_t(n) * (c + 1) / chunks, m = b - a;
        cudaStream_t s_cast = s->pipe[2 + c % VX_PIPE_CAST_STREAMS];
        e = cudaMemcpyAsync(dr + a, rh + a * sizeof(vx_ray), m * sizeof(vx_ray), cudaMemcpyHostToDevice, s_in);
        if (e == cudaSuccess) e = cudaEventRecord(s->pipe_in[c], s_in);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s_cast, s->pipe_in[c], 0);
        if (e != cudaSuccess) return vx::cuda_fail(e, w + ": copy in");
        int r = vx::launch_cast(s->dev, dr + a, uint32_t(m), tmin, tmax, dh + a, dc ? dc + a * colw : nullptr, nullptr,
                                s_cast, lod);
        if (r != 0) return vx::cuda_fail(cudaError_t(r), w + ": launch");
        e = cudaEventRecord(s->pipe_cast[c], s_cast);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s_out, s->pipe_cast[c], 0);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(hh + a * sizeof(vx_hit), dh + a, m * sizeof(vx_hit), cudaMemcpyDeviceToHost, s_out);
        if (e == cudaSuccess && dc)
            e = cudaMemcpyAsync(ch + a * colw, dc + a * colw, m * colw, cudaMemcpyDeviceToHost, s_out);
        if (e != cudaSuccess) return vx::cuda_fail(e, w + ": copy out");
    }
    for (int i = 1; i < 2 + VX_PIPE_CAST_STREAMS && e == cudaSuccess; ++i) e = cudaStreamSynchronize(s->pipe[i]);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s_in);
    if (e != cudaSuccess) return vx::cuda_fail(e, w + ": synchronize");
    return VX_OK;
}

}  // namespace

int vx_cast_rays(const vx_scene* s, const vx_ray* rays, uint32_t n, float tmin, float tmax, vx_hit* hits,
                 void* color, vx_ray_counters* counters, void* stream) {
    return cast_rays_dev("vx_cast_rays", s, rays, n, tmin, tmax, nullptr, hits, color, counters, stream);
}

int vx_cast_shadow_rays(const vx_scene* cs, const vx_ray* rays, const vx_hit* hits, uint32_t n,
                        const float light_dir[3], float tmin, float tmax, vx_hit* shadow_hits, void* stream) {
    return vx::guarded("vx_cast_shadow_rays", [&]() -> int {
        if (!cs || !light_dir || (n && (!rays || !hits || !shadow_hits)))
            return fail(VX_EINVAL, "vx_cast_shadow_rays: null argument");
        if (reinterpret_cast<uintptr_t>(rays) % 8 || reinterpret_cast<uintptr_t>(hits) % 16 ||
            reinterpret_cast<uintptr_t>(shadow_hits) % 16)
            return fail(VX_EINVAL, "vx_cast_shadow_rays: misaligned buffer");
        if (std::isnan(tmin) || std::isnan(tmax)) return fail(VX_EINVAL, "vx_cast_shadow_rays: t_min / t_max is NaN");
        if (n == 0) return VX_OK;
        vx_scene* s = const_cast<vx_scene*>(cs);
        int dev = -1;
        cudaGetDevice(&dev);
        if (dev != s->device) return fail(VX_EINVAL, "vx_cast_shadow_rays: the scene belongs to another device");
        std::lock_guard<std::mutex> lk(s->stage_mu);
        const uint64_t need = vx::shadow_scratch_bytes(n);
        if (need > s->shadow_bytes) {
            if (s->shadow) cudaFree(s->shadow);
            s->shadow = nullptr;
            s->shadow_bytes = 0;
            const cudaError_t e = cudaMalloc(&s->shadow, need);
            if (e != cudaSuccess) return vx::cuda_fail(e, "vx_cast_shadow_rays: cudaMalloc");
            s->shadow_bytes = need;
        }
        vx_ray* crays = nullptr;
        uint32_t* map = nullptr;
        uint32_t* count = nullptr;
        int r = vx::launch_shadow_compact(rays, hits, n, light_dir, s->shadow, &crays, &map, &count, shadow_hits, stream);
        if (r != 0) return vx::cuda_fail(cudaError_t(r), "vx_cast_shadow_rays: compaction launch");
        r = vx::launch_cast_mapped(s->dev, crays, n, count, map, tmin, tmax, shadow_hits, stream);
        if (r != 0) return vx::cuda_fail(cudaError_t(r), "vx_cast_shadow_rays: launch");
        return VX_OK;
    });
}

int vx_cast_rays_lod(const vx_scene* s, const vx_ray* rays, uint32_t n, float tmin, float tmax,
                     const vx_lod_params* lod, vx_hit* hits, void* color, vx_ray_counters* counters, void* stream) {
    if (!lod) return fail(VX_EINVAL, "vx_cast_rays_lod: null LOD parameters");
    return cast_rays_dev("vx_cast_rays_lod", s, rays, n, tmin, tmax, lod, hits, color, counters, stream);
}

int vx_cast_rays_host(const vx_scene* s, const vx_ray* rays_host, uint32_t n, float tmin, float tmax,
                      vx_hit* hits_host, void* color_host, void* stream) {
    return cast_rays_host("vx_cast_rays_host", s, rays_host, n, tmin, tmax, nullptr, hits_host, color_host, stream);
}

int vx_cast_rays_host_lod(const vx_scene* s, const vx_ray* rays_host, uint32_t n, float tmin, float tmax,
                          const vx_lod_params* lod, vx_hit* hits_host, void* color_host, void* stream) {
    if (!lod) return fail(VX_EINVAL, "vx_cast_rays_host_lod: null LOD parameters");
    return cast_rays_host("vx_cast_rays_host_lod", s, rays_host, n, tmin, tmax, lod, hits_host, color_host, stream);
}

int vx_lod_from_camera(float fov_y, int32_t screen_height, float near_plane, vx_lod_params* out) {
    if (!out || screen_height <= 0) return fail(VX_EINVAL, "vx_lod_from_camera: bad argument");
    // pixel angle = fovY / H; cone spread = 2 tan(angle / 2) (SVOLOD.h:83-119)
    const float pixel_angle = fov_y / static_cast<float>(screen_height);
    const float dir = 2.0f * ::tanf(pixel_angle * 0.5f);
    out->ray_dir_size = dir;
    out->ray_orig_size = near_plane * dir;
    return VX_OK;
}

int vx_lod_with_bias(const vx_lod_params* in, float bias, vx_lod_params* out) {
    if (!in || !out) return fail(VX_EINVAL, "vx_lod_with_bias: null argument");
    const float m = ::powf(2.0f, bias);
    const vx_lod_params r{in->ray_orig_size * m, in->ray_dir_size * m};
    *out = r;
    return VX_OK;
}

int vx_render(const vx_scene* s, const vx_camera_pc* pc, uint32_t w, uint32_t h, uint32_t* image, vx_hit* hits,
              void* color, void* stream) {
    if (!s || !pc) return fail(VX_EINVAL, "vx_render: null argument");
    if (uint64_t(w) * h > 0xFFFFFFFFull) return fail(VX_EOVERFLOW, "vx_render: width * height exceeds 2^32");
    if (reinterpret_cast<uintptr_t>(hits) % 16 || reinterpret_cast<uintptr_t>(image) % 4 ||
        reinterpret_cast<uintptr_t>(color) % 4)
        return fail(VX_EINVAL, "vx_render: misaligned output");
    const vx::CameraDev cam = vx::camera_from_pc(*pc);
    int r = vx::launch_render(s->dev, cam, w, h, image, hits, color, stream);
    if (r != 0) return vx::cuda_fail(cudaError_t(r), "vx_render: launch");
    return VX_OK;
}

int vx_camera_rays(const vx_camera_pc* pc, uint32_t w, uint32_t h, vx_ray* rays) {
    if (!pc || (uint64_t(w) * h != 0 && !rays)) return fail(VX_EINVAL, "vx_camera_rays: null argument");
    if (uint64_t(w) * h > 0xFFFFFFFFull) return fail(VX_EOVERFLOW, "vx_camera_rays: width * height exceeds 2^32");
    const vx::CameraDev cam = vx::camera_from_pc(*pc);
    for (uint32_t y = 0; y < h; ++y)
        for (uint32_t x = 0; x < w; ++x) vx::camera_ray(cam, x, y, w, h, rays[uint64_t(y) * w + x], nullptr);
    return VX_OK;
}

int vx_camera_rays_dev(const vx_camera_pc* pc, uint32_t w, uint32_t h, vx_ray* rays, void* stream) {
    if (!pc || (uint64_t(w) * h != 0 && !rays)) return fail(VX_EINVAL, "vx_camera_rays_dev: null argument");
    if (uint64_t(w) * h > 0xFFFFFFFFull) return fail(VX_EOVERFLOW, "vx_camera_rays_dev: width * height exceeds 2^32");
    const vx::CameraDev cam = vx::camera_from_pc(*pc);
    int r = vx::launch_camera_rays(cam, w, h, rays, stream);
    if (r != 0) return vx::cuda_fail(cudaError_t(r), "vx_camera_rays_dev: launch");
    return VX_OK;
}

}  // extern "C"
