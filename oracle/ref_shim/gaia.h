// Stand-in for the gaia-ecs header the reference's SVO path includes
// (gaia::ecs::Entity, gaia::ecs::World, GAIA_LAYOUT), written for this test
// build only (TEST INFRASTRUCTURE ONLY; see oracle/ref_build.sh).  The world
// is a map from entity to its components, enough for the component reads the
// ray-cast path makes (GaiaVoxelWorld::getComponentValue).
#pragma once

#include <any>
#include <cstdint>
#include <stdexcept>
#include <typeindex>
#include <unordered_map>

#define GAIA_LAYOUT(x) static constexpr int gaia_layout_unused = 0

namespace gaia::ecs {

struct Entity {
    uint64_t v = ~uint64_t(0);  // the default entity is the invalid one
    Entity() = default;
    explicit Entity(uint64_t id) : v(id) {}
    uint64_t id() const { return v; }
    uint64_t value() const { return v; }
    bool operator==(const Entity& o) const { return v == o.v; }
    bool operator!=(const Entity& o) const { return v != o.v; }
};

struct Component {};

class World {
public:
    bool valid(Entity e) const { return e.v != ~uint64_t(0) && comps_.count(e.v) != 0; }
    template <class T>
    bool has(Entity e) const {
        auto it = comps_.find(e.v);
        return it != comps_.end() && it->second.count(std::type_index(typeid(T))) != 0;
    }
    template <class T>
    const T& get(Entity e) const {
        return std::any_cast<const T&>(comps_.at(e.v).at(std::type_index(typeid(T))));
    }
    template <class T>
    T& get(Entity e) {
        return std::any_cast<T&>(comps_.at(e.v).at(std::type_index(typeid(T))));
    }
    template <class T>
    void add(Entity e, const T& value) {
        comps_[e.v][std::type_index(typeid(T))] = value;
    }
    void touch(Entity e) { comps_[e.v]; }

private:
    std::unordered_map<uint64_t, std::unordered_map<std::type_index, std::any>> comps_;
};

}  // namespace gaia::ecs

namespace std {
template <>
struct hash<gaia::ecs::Entity> {
    size_t operator()(const gaia::ecs::Entity& e) const { return std::hash<uint64_t>()(e.v); }
};
}  // namespace std
