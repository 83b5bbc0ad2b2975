// vx_octree.hpp - C++ facade over the C ABI (vx.h) with the shape of the
// reference's query interface, ISVOStructure::castRay
// (SVO/include/ISVOStructure.h:101-126) and LaineKarrasOctree::castRay
// (SVO/src/SVOTraversal.cpp:189-196): a single ray returns a RayHit with
// hit / tMin / tMax / hitPoint / normal / scale and the hit voxel's integer
// position in place of the ECS entity.  castRays() casts a batch in one call.
// castRayWithLOD / castRayLOD / castRayScreenSpaceLOD and LODParameters follow
// SVOTraversal.cpp:198-232 and SVO/include/SVOLOD.h:50-177.
//
// Header-only; link with libvx.so.  No glm dependency: positions are float[3].
#pragma once

#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "vx.h"

namespace vx {

struct Vec3 {
    float x = 0, y = 0, z = 0;
};

// ISVOStructure::RayHit (ISVOStructure.h:101-112) without the ECS handle.
struct RayHit {
    bool hit = false;
    float tMin = 0.0f;       // distance along the normalised direction
    float tMax = 0.0f;       // tMin + voxel size (1; the cell size for an LOD hit)
    Vec3 hitPoint;           // origin + normalize(direction) * tMin
    Vec3 normal;             // entry face, +-1 on one axis; +y for an LOD hit
    int scale = 0;           // maxLevels - 1; the cell's user scale for an LOD hit
    uint32_t brick = 0xFFFFFFFFu;  // 0xFFFFFFFF for an LOD hit (no entity)
    uint32_t voxel = 0xFFFFu;  // z*64 + y*8 + x within the brick
    uint32_t node = 0xFFFFFFFFu;
    int32_t voxelPos[3] = {0, 0, 0};  // integer position of the hit voxel (the entity's key)
    uint8_t flags = 0;
};

// LODParameters (SVOLOD.h:50-177).
struct LODParameters {
    float rayOrigSize = 0.0f;  // cone diameter at the origin
    float rayDirSize = 0.0f;   // cone growth per unit distance; 0 disables the cut

    static LODParameters fromCamera(float fovY, int screenHeight) {
        return fromCameraWithNearPlane(fovY, screenHeight, 0.0f);
    }
    static LODParameters fromCameraWithNearPlane(float fovY, int screenHeight, float nearPlane) {
        vx_lod_params p{};
        if (vx_lod_from_camera(fovY, screenHeight, nearPlane, &p) != VX_OK)
            throw std::invalid_argument(vx_last_error_string());
        return {p.ray_orig_size, p.ray_dir_size};
    }
    float getProjectedPixelSize(float voxelDistance) const { return voxelDistance * rayDirSize + rayOrigSize; }
    bool shouldTerminate(float voxelDistance, float voxelSize) const {
        return getProjectedPixelSize(voxelDistance) >= voxelSize;
    }
    bool isEnabled() const { return rayDirSize > 0.0f; }
    LODParameters withBias(float bias) const {
        const vx_lod_params in{rayOrigSize, rayDirSize};
        vx_lod_params p{};
        vx_lod_with_bias(&in, bias, &p);
        return {p.ray_orig_size, p.ray_dir_size};
    }
};

class Error : public std::runtime_error {
public:
    Error(int status, const std::string& what) : std::runtime_error(what), status(status) {}
    int status;
};

inline void check(int status) {
    if (status != VX_OK) throw Error(status, vx_last_error_string());
}

// A scene resident on the current CUDA device plus the host copy of its brick
// coordinates (needed to turn (brick, voxel) into a voxel position).
class CudaOctree {
public:
    explicit CudaOctree(const vx_scene_desc& desc) : cfg_(desc.config) {
        check(vx_scene_create(&desc, &scene_));
        coord_.assign(desc.brick_coord, desc.brick_coord + desc.brick_count);
    }
    CudaOctree(const CudaOctree&) = delete;
    CudaOctree& operator=(const CudaOctree&) = delete;
    ~CudaOctree() { vx_scene_destroy(scene_); }

    vx_scene* handle() const { return scene_; }
    int getMaxLevels() const { return cfg_.max_levels; }

    // LaineKarrasOctree::castRay(origin, direction, tMin, tMax).
    RayHit castRay(const Vec3& origin, const Vec3& direction, float tMin = 0.0f,
                   float tMax = 3.402823466e+38f) const {
        vx_ray r{origin.x, origin.y, origin.z, direction.x, direction.y, direction.z};
        vx_hit h{};
        check(vx_cast_rays_host(scene_, &r, 1, tMin, tMax, &h, nullptr, nullptr));
        return toRayHit(r, h);
    }

    // LaineKarrasOctree::castRayWithLOD(origin, direction, lodParams, tMin, tMax).
    RayHit castRayWithLOD(const Vec3& origin, const Vec3& direction, const LODParameters& lod,
                          float tMin = 0.0f, float tMax = 3.402823466e+38f) const {
        vx_ray r{origin.x, origin.y, origin.z, direction.x, direction.y, direction.z};
        vx_hit h{};
        const vx_lod_params p{lod.rayOrigSize, lod.rayDirSize};
        check(vx_cast_rays_host_lod(scene_, &r, 1, tMin, tMax, &p, &h, nullptr, nullptr));
        return toRayHit(r, h);
    }
    // castRayLOD(origin, direction, lodBias, ...): the bias is the cone spread.
    RayHit castRayLOD(const Vec3& origin, const Vec3& direction, float lodBias, float tMin = 0.0f,
                      float tMax = 3.402823466e+38f) const {
        return castRayWithLOD(origin, direction, LODParameters{0.0f, lodBias}, tMin, tMax);
    }
    // castRayScreenSpaceLOD(origin, direction, fovY, screenHeight, ...).
    RayHit castRayScreenSpaceLOD(const Vec3& origin, const Vec3& direction, float fovY, int screenHeight,
                                 float tMin = 0.0f, float tMax = 3.402823466e+38f) const {
        return castRayWithLOD(origin, direction, LODParameters::fromCamera(fovY, screenHeight), tMin, tMax);
    }

    // Batch form: one host->device copy, one launch, one copy back.
    std::vector<RayHit> castRays(const std::vector<vx_ray>& rays, float tMin = 0.0f,
                                 float tMax = 3.402823466e+38f, const LODParameters* lod = nullptr) const {
        std::vector<vx_hit> hits(rays.size());
        if (!rays.empty()) {
            if (lod) {
                const vx_lod_params p{lod->rayOrigSize, lod->rayDirSize};
                check(vx_cast_rays_host_lod(scene_, rays.data(), uint32_t(rays.size()), tMin, tMax, &p, hits.data(),
                                            nullptr, nullptr));
            } else {
                check(vx_cast_rays_host(scene_, rays.data(), uint32_t(rays.size()), tMin, tMax, hits.data(),
                                        nullptr, nullptr));
            }
        }
        std::vector<RayHit> out(rays.size());
        for (size_t i = 0; i < rays.size(); ++i) out[i] = toRayHit(rays[i], hits[i]);
        return out;
    }

private:
    RayHit toRayHit(const vx_ray& r, const vx_hit& h) const {
        RayHit o;
        o.flags = h.flags;
        if (!(h.flags & VX_HIT_HIT)) return o;
        o.hit = true;
        o.tMin = h.t;
        o.tMax = h.t + 1.0f;
        const float dd = (r.dx * r.dx + r.dy * r.dy) + r.dz * r.dz;
        const float inv = 1.0f / std::sqrt(dd);
        if (h.brick == 0xFFFFFFFFu) {
            // LOD hit (SVOTraversal.cpp:639-649): hitPoint = origin + dir * t,
            // tMax = t + 2^(scale - maxLevels) * worldSize.x, normal +y.
            const float size = std::ldexp(1.0f, int(h.scale) - cfg_.max_levels) *
                               (cfg_.world_max[0] - cfg_.world_min[0]);
            o.tMax = h.t + size;
            o.hitPoint = {r.ox + (r.dx * inv) * h.t, r.oy + (r.dy * inv) * h.t, r.oz + (r.dz * inv) * h.t};
            o.normal = {0.0f, 1.0f, 0.0f};
            o.scale = h.scale;
            o.node = h.node;
            return o;
        }
        // hitPoint in local space, then back to world (SVOBrickDDA.cpp:508, 174)
        o.hitPoint = {((r.ox + (0.0f - cfg_.world_min[0])) + (r.dx * inv) * h.t) + cfg_.world_min[0],
                      ((r.oy + (0.0f - cfg_.world_min[1])) + (r.dy * inv) * h.t) + cfg_.world_min[1],
                      ((r.oz + (0.0f - cfg_.world_min[2])) + (r.dz * inv) * h.t) + cfg_.world_min[2]};
        const int axis = (h.flags & VX_HIT_AXIS_MASK) >> 1;
        const float s = (h.flags & VX_HIT_NORMAL_NEG) ? -1.0f : 1.0f;
        o.normal = {axis == 0 ? s : 0.0f, axis == 1 ? s : 0.0f, axis == 2 ? s : 0.0f};
        o.scale = h.scale;
        o.brick = h.brick;
        o.voxel = h.voxel;
        o.node = h.node;
        const uint32_t c = coord_[h.brick];
        const int q[3] = {int(std::floor(cfg_.world_min[0])), int(std::floor(cfg_.world_min[1])),
                          int(std::floor(cfg_.world_min[2]))};
        o.voxelPos[0] = int(c & 0x3FF) * 8 + int(h.voxel & 7) + q[0];
        o.voxelPos[1] = int((c >> 10) & 0x3FF) * 8 + int((h.voxel >> 3) & 7) + q[1];
        o.voxelPos[2] = int((c >> 20) & 0x3FF) * 8 + int(h.voxel >> 6) + q[2];
        return o;
    }

    vx_octree_config cfg_;
    vx_scene* scene_ = nullptr;
    std::vector<uint32_t> coord_;
};

}  // namespace vx
