// vx_octree.hpp - C++ facade over the C ABI (vx.h) with the shape of the
// reference's query interface, ISVOStructure::castRay
// (SVO/include/ISVOStructure.h:101-126) and LaineKarrasOctree::castRay
// (SVO/src/SVOTraversal.cpp:189-196): a single ray returns a RayHit with
// hit / tMin / tMax / hitPoint / normal / scale and the hit voxel's integer
// position in place of the ECS entity.  castRays() casts a batch in one call.
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
    float tMax = 0.0f;       // tMin + voxel size (1)
    Vec3 hitPoint;           // origin + normalize(direction) * tMin
    Vec3 normal;             // entry face, +-1 on one axis
    int scale = 0;           // maxLevels - 1
    uint32_t brick = 0xFFFFFFFFu;
    uint32_t voxel = 0xFFFFu;  // z*64 + y*8 + x within the brick
    uint32_t node = 0xFFFFFFFFu;
    int32_t voxelPos[3] = {0, 0, 0};  // integer position of the hit voxel (the entity's key)
    uint8_t flags = 0;
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

    // Batch form: one host->device copy, one launch, one copy back.
    std::vector<RayHit> castRays(const std::vector<vx_ray>& rays, float tMin = 0.0f,
                                 float tMax = 3.402823466e+38f) const {
        std::vector<vx_hit> hits(rays.size());
        if (!rays.empty())
            check(vx_cast_rays_host(scene_, rays.data(), uint32_t(rays.size()), tMin, tMax, hits.data(),
                                    nullptr, nullptr));
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
        // hitPoint in local space, then back to world (SVOBrickDDA.cpp:508, 174)
        o.hitPoint = {((r.ox + (0.0f - cfg_.world_min[0])) + (r.dx * inv) * h.t) + cfg_.world_min[0],
                      ((r.oy + (0.0f - cfg_.world_min[1])) + (r.dy * inv) * h.t) + cfg_.world_min[1],
                      ((r.oz + (0.0f - cfg_.world_min[2])) + (r.dz * inv) * h.t) + cfg_.world_min[2]};
        const int axis = (h.flags & VX_HIT_AXIS_MASK) >> 1;
        const float s = (h.flags & VX_HIT_NORMAL_NEG) ? -1.0f : 1.0f;
        o.normal = {axis == 0 ? s : 0.0f, axis == 1 ? s : 0.0f, axis == 2 ? s : 0.0f};
        o.scale = cfg_.max_levels - 1;
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
