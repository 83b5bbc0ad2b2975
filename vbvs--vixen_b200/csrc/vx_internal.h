// vx_internal.h - shared between the host API (vx_api.cpp, vx_build.cpp)
// and the CUDA kernels (vx_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <exception>
#include <new>
#include <string>

#include "../../include/vx.h"

namespace vx {

// Scene as the kernels see it (passed by value as a kernel parameter).
struct DevScene {
    float wmin[3], wmax[3], wsize[3];  // wsize = wmax - wmin (float subtract)
    float wsm[3];                      // wsize - 0.001 (SVOBrickDDA.cpp:128, 143)
    float wrl;                         // length(wsize), worldRayLength (SVOTraversal.cpp:552)
    float wsinv[3];                    // 1 / wsize where that is exact (power-of-two size), else 0
    int32_t qwm[3];                    // floor(world_min), VoxelComponents.h:373-379
    int32_t max_levels;
    int32_t min_scale;                 // 22 - max_levels + 1
    int32_t brick_user_scale;          // max_levels - brick_depth (SVOTraversal.cpp:305)
    int32_t bpa;                       // bricks per axis
    uint32_t node_count, brick_count;
    const uint2* nodes;                // {child_ptr, valid | leaf << 8}
    const uint32_t* node_brick;
    const uint32_t* grid;              // bpa^3
    const uint32_t* coord;             // brick grid coordinate, 10:10:10
    const uint4* occ;                  // 4 x uint4 (16 words) per brick
    int32_t color_kind;
    const uint32_t* rgba;              // 512 per brick
    const uint2* dxt;                  // 32 per brick
    const uint4* nrm;                  // DXT normal blocks, 32 per brick, or null
};

// Accessors of an opaque vx_scene (vx_api.cpp).
const DevScene& scene_dev(const vx_scene* s);
int scene_device(const vx_scene* s);

// Device slices of a new scene's pool and their sizes in bytes.
struct ScenePool {
    void *nodes, *node_brick, *grid, *coord, *occ, *color, *nrm;
    uint64_t sz_nodes, sz_nb, sz_grid, sz_coord, sz_occ, sz_color, sz_nrm;
};
// Allocates a scene on the current device for the given counts and fills its
// device view; the caller writes the slices (vx_scene_destroy frees it).
int scene_alloc(const vx_octree_config& c, uint32_t node_count, uint32_t brick_count, int32_t color_kind,
                bool normals, vx_scene** out, ScenePool* p);
int cuda_fail(cudaError_t e, const std::string& what);

// Violation words of the bounds-checked build, one per translation unit with
// device code (read and cleared; 0 in the default build).
uint32_t violations_kernels();
uint32_t violations_batch();
uint32_t violations_diff();
uint32_t violations_payload();

// Per-thread-local error string.
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);

// Runs an entry point's body and turns a C++ exception (an allocation or a
// thread that could not be made) into a status: no exception crosses the ABI.
template <class F>
int guarded(const char* what, F&& body) noexcept {
    try {
        return body();
    } catch (const std::bad_alloc&) {
        return fail(VX_ENOMEM, std::string(what) + ": out of host memory");
    } catch (const std::exception& e) {
        return fail(VX_EINVAL, std::string(what) + ": " + e.what());
    } catch (...) {
        return fail(VX_EINVAL, std::string(what) + ": unexpected exception");
    }
}

// Kernel launchers (vx_kernels.cu).  Return cudaError_t as int.
// lod: nullptr, or LODParameters {ray_orig_size, ray_dir_size} with ray_dir_size > 0.
int launch_cast(const DevScene& s, const vx_ray* rays, uint32_t n, float tmin, float tmax,
                vx_hit* hits, void* color, vx_ray_counters* counters, void* stream,
                const vx_lod_params* lod = nullptr);
struct CameraDev {
    float pos[3], dir[3], up[3], right[3];
    float aspect, tan_half_fov;
};
int launch_render(const DevScene& s, const CameraDev& cam, uint32_t w, uint32_t h, uint32_t* image,
                  vx_hit* hits, void* color, void* stream);
int launch_camera_rays(const CameraDev& cam, uint32_t w, uint32_t h, vx_ray* rays, void* stream);
// cast of device-compacted rays: min(n_max, *count) rays, ray i's record to slot map[i]
int launch_cast_mapped(const DevScene& s, const vx_ray* rays, uint32_t n_max, const uint32_t* count,
                       const uint32_t* map, float tmin, float tmax, vx_hit* hits, void* stream);

// Shadow-ray compaction (vx_batch.cu): scratch bytes for n primary rays, and
// the launches that fill it (compacted rays, their slots, the device-side
// count) and write the invalid record into the slots of primary misses.
uint64_t shadow_scratch_bytes(uint32_t n);
int launch_shadow_compact(const vx_ray* rays, const vx_hit* hits, uint32_t n, const float light_dir[3], void* scratch,
                          vx_ray** out_rays, uint32_t** map, uint32_t** count, vx_hit* shadow_hits, void* stream);

// Host camera setup shared by vx_render and vx_camera_rays: tan(radians(fov/2))
// is evaluated once on the host (RayGeneration.glsl:62).
CameraDev camera_from_pc(const vx_camera_pc& pc);

}  // namespace vx
