// The parts of the reference's GaiaVoxelWorld that its rebuild and ray cast
// call, over the gaia stand-in (gaia.h here), plus the C entry points of the
// reference build (oracle/_ref/libvx_ref.so).  TEST INFRASTRUCTURE ONLY: the
// tests compare the oracle (oracle/vx_oracle.cpp) with the reference's own
// LaineKarrasOctree::rebuild and castRay compiled from its sources by
// oracle/ref_build.sh.
//
// What this file restates (GaiaVoxel/src/GaiaVoxelWorld.cpp, by behaviour):
// a voxel is an entity with a MortonKey (MortonKeyUtils::fromPosition of its
// position) and the components of its creation request; the Morton index maps
// a key to its entity; querySolidVoxels returns, in creation order, the
// entities without a Density or with Density > 0; queryRegion the entities
// whose key position lies in the closed box; getEntityByWorldSpace /
// getEntityByMorton look a key up; countBrickEntities counts the keys of a
// brick.  The ECS storage is the stand-in's map, not gaia's archetypes.
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "ComponentData.h"
#include "GaiaVoxelWorld.h"
#include "LaineKarrasOctree.h"
#include "MortonEncoding.h"
#include "VoxelComponents.h"

namespace Vixen::GaiaVoxel {

struct GaiaVoxelWorld::Impl {
    gaia::ecs::World world;
    std::unordered_map<uint64_t, gaia::ecs::Entity> mortonIndex;
    std::vector<gaia::ecs::Entity> order;  // creation order (the query order)
    uint64_t next = 1;
};

GaiaVoxelWorld::GaiaVoxelWorld() : m_impl(std::make_unique<Impl>()) {}
GaiaVoxelWorld::~GaiaVoxelWorld() = default;

GaiaVoxelWorld::EntityID GaiaVoxelWorld::createVoxel(const VoxelCreationRequest& request) {
    gaia::ecs::Entity e(m_impl->next++);
    m_impl->world.touch(e);
    const MortonKey key = MortonKeyUtils::fromPosition(request.position);
    m_impl->world.add<MortonKey>(e, key);
    for (const auto& req : request.components)
        std::visit(
            [&](auto&& c) {
                using T = std::decay_t<decltype(c)>;
                if constexpr (!std::is_same_v<T, MortonKey> && !std::is_same_v<T, std::monostate>)
                    m_impl->world.add<T>(e, c);
            },
            req.component);
    m_impl->mortonIndex[key.code] = e;
    m_impl->order.push_back(e);
    return e;
}

const gaia::ecs::World& GaiaVoxelWorld::getWorld() const { return m_impl->world; }
gaia::ecs::World& GaiaVoxelWorld::getWorld() { return m_impl->world; }

std::optional<glm::vec3> GaiaVoxelWorld::getPosition(EntityID id) const {
    if (!m_impl->world.valid(id) || !m_impl->world.has<MortonKey>(id)) return std::nullopt;
    return MortonKeyUtils::toWorldPos(m_impl->world.get<MortonKey>(id));
}

std::vector<GaiaVoxelWorld::EntityID> GaiaVoxelWorld::queryRegion(const glm::vec3& lo, const glm::vec3& hi) const {
    std::vector<EntityID> out;
    for (const auto& e : m_impl->order) {
        const glm::vec3 p = MortonKeyUtils::toWorldPos(m_impl->world.get<MortonKey>(e));
        if (p.x >= lo.x && p.x <= hi.x && p.y >= lo.y && p.y <= hi.y && p.z >= lo.z && p.z <= hi.z) out.push_back(e);
    }
    return out;
}

std::vector<GaiaVoxelWorld::EntityID> GaiaVoxelWorld::querySolidVoxels() const {
    std::vector<EntityID> out;
    for (const auto& e : m_impl->order)
        if (!m_impl->world.has<Density>(e) || m_impl->world.get<Density>(e).value > 0.0f) out.push_back(e);
    return out;
}

GaiaVoxelWorld::EntityID GaiaVoxelWorld::getEntityByWorldSpace(glm::vec3 worldPos) const {
    const auto it = m_impl->mortonIndex.find(MortonKeyUtils::fromPosition(worldPos).code);
    return it != m_impl->mortonIndex.end() ? it->second : EntityID{};
}

GaiaVoxelWorld::EntityID GaiaVoxelWorld::getEntityByMorton(uint64_t code) const {
    const auto it = m_impl->mortonIndex.find(code);
    return it != m_impl->mortonIndex.end() ? it->second : EntityID{};
}

GaiaVoxelWorld::EntityID GaiaVoxelWorld::getEntityByMorton(const Vixen::Core::MortonCode64& m) const {
    return getEntityByMorton(m.code);
}

uint32_t GaiaVoxelWorld::countBrickEntities(const Vixen::Core::MortonCode64& base, uint32_t size) const {
    uint32_t n = 0;
    for (uint32_t z = 0; z < size; ++z)
        for (uint32_t y = 0; y < size; ++y)
            for (uint32_t x = 0; x < size; ++x)
                if (m_impl->mortonIndex.count(base.addLocalOffset(x, y, z).code)) ++n;
    return n;
}

}  // namespace Vixen::GaiaVoxel

// Unreached members of the reference's attribute registry (the cast runs with
// registry == nullptr, so only its ECS branch executes).
namespace Vixen::VoxelData {
BrickView AttributeRegistry::getBrick(uint32_t) { throw std::runtime_error("attribute registry not built"); }
std::any* BrickView::getKeyAttributePointer() const { throw std::runtime_error("attribute registry not built"); }
}  // namespace Vixen::VoxelData

// ---------------------------------------------------------------------------
// C entry points
// ---------------------------------------------------------------------------
namespace {

struct RefScene {
    Vixen::GaiaVoxel::GaiaVoxelWorld world;
    std::unique_ptr<Vixen::SVO::LaineKarrasOctree> octree;
};

// The fields of the reference's RayHit (SVO/include/ISVOStructure.h:101-112),
// the entity given by its position (-1 when the hit carries no entity).
struct RefHit {
    float t, t_exit, hit_point[3], normal[3];
    int32_t hit, scale;
    float entity_pos[3];
};

}  // namespace

extern "C" {

// Voxels created at world positions (x, y, z) with Density 1 (the reference
// keys each by MortonKeyUtils::fromPosition) in a world [wmin, wmax]^3, then
// LaineKarrasOctree::rebuild.  Returns NULL and a message on failure.
// materials (may be NULL): a Material component per voxel, which the
// rebuild's compressed colour payload reads (MaterialIdToColor).
void* vxr_build(const float* positions, uint64_t n, const float wmin[3], const float wmax[3], int max_levels,
                const uint32_t* materials, char* err, int errlen) {
    try {
        auto s = std::make_unique<RefScene>();
        using namespace Vixen::GaiaVoxel;
        for (uint64_t i = 0; i < n; ++i) {
            const glm::vec3 p(positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]);
            const ComponentQueryRequest comps[2] = {ComponentQueryRequest(Density{1.0f}),
                                                    ComponentQueryRequest(Material{materials ? materials[i] : 0u})};
            s->world.createVoxel(VoxelCreationRequest(p, std::span<const ComponentQueryRequest>(comps, materials ? 2 : 1)));
        }
        s->octree = std::make_unique<Vixen::SVO::LaineKarrasOctree>(s->world, nullptr, max_levels, 3);
        s->octree->rebuild(s->world, glm::vec3(wmin[0], wmin[1], wmin[2]), glm::vec3(wmax[0], wmax[1], wmax[2]));
        return s.release();
    } catch (const std::exception& e) {
        if (err && errlen > 0) {
            std::strncpy(err, e.what(), size_t(errlen) - 1);
            err[errlen - 1] = 0;
        }
        return nullptr;
    }
}

void vxr_free(void* h) { delete static_cast<RefScene*>(h); }

uint32_t vxr_node_count(void* h) {
    const auto* o = static_cast<RefScene*>(h)->octree->getOctree();
    return (o && o->root) ? uint32_t(o->root->childDescriptors.size()) : 0u;
}

// The reference's descriptors as 64-bit ChildDescriptor words.
void vxr_descriptors(void* h, uint64_t* out) {
    const auto* o = static_cast<RefScene*>(h)->octree->getOctree();
    const auto& d = o->root->childDescriptors;
    static_assert(sizeof(d[0]) == 8, "ChildDescriptor is 8 bytes");
    if (!d.empty()) std::memcpy(out, d.data(), d.size() * 8);
}

uint32_t vxr_brick_count(void* h) {
    const auto* o = static_cast<RefScene*>(h)->octree->getOctree();
    return (o && o->root) ? uint32_t(o->root->brickViews.size()) : 0u;
}

// The rebuild's brick payloads: DXT1 colours (32 u64 per brick), DXT normals
// (32 x {blockA, blockB} per brick) and material words (512 u32 per brick).
void vxr_payloads(void* h, uint64_t* colors, uint64_t* normals, uint32_t* materials) {
    const auto& r = *static_cast<RefScene*>(h)->octree->getOctree()->root;
    if (colors && !r.compressedColors.empty()) std::memcpy(colors, r.compressedColors.data(), r.compressedColors.size() * 8);
    for (size_t i = 0; normals && i < r.compressedNormals.size(); ++i) {
        normals[2 * i] = r.compressedNormals[i].blockA;
        normals[2 * i + 1] = r.compressedNormals[i].blockB;
    }
    if (materials && !r.brickMaterialData.empty())
        std::memcpy(materials, r.brickMaterialData.data(), r.brickMaterialData.size() * 4);
}

// castRay over n rays {origin, direction}; with lod (rayOrigSize, rayDirSize)
// castRayWithLOD.
void vxr_cast_rays(void* h, const float* rays, uint64_t n, float tmin, float tmax, const float* lod, RefHit* out) {
    const auto& oct = *static_cast<RefScene*>(h)->octree;
    for (uint64_t i = 0; i < n; ++i) {
        const float* r = rays + 6 * i;
        const glm::vec3 org(r[0], r[1], r[2]), dir(r[3], r[4], r[5]);
        const auto hit = lod ? oct.castRayWithLOD(org, dir, Vixen::SVO::LODParameters(lod[0], lod[1]), tmin, tmax)
                             : oct.castRay(org, dir, tmin, tmax);
        RefHit& o = out[i];
        o.hit = hit.hit ? 1 : 0;
        o.t = hit.tMin;
        o.t_exit = hit.tMax;
        o.scale = hit.scale;
        for (int a = 0; a < 3; ++a) {
            o.hit_point[a] = hit.hitPoint[a];
            o.normal[a] = hit.normal[a];
        }
        o.entity_pos[0] = o.entity_pos[1] = o.entity_pos[2] = -1.0f;
        if (hit.hit) {
            if (auto p = static_cast<RefScene*>(h)->world.getPosition(hit.entity)) {
                o.entity_pos[0] = p->x;
                o.entity_pos[1] = p->y;
                o.entity_pos[2] = p->z;
            }
        }
    }
}

}  // extern "C"
