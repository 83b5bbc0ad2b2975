// Exercises the C++ facade (include/vx_octree.hpp) the way the reference's
// tests call LaineKarrasOctree::castRay: voxels at (17, 3, 10), (0, 0, 0) and
// (63, 63, 63) in a 64^3 grid (the corner voxels make the octree root span
// the whole grid), rays along +x, -y and a diagonal.  Prints one line per ray.
#include <cstdio>
#include <vector>

#include "vx_octree.hpp"

int main() {
    const uint32_t R = 64;
    std::vector<uint64_t> bits(R * R * (R / 64), 0);
    auto set = [&](int x, int y, int z) { bits[(size_t(z) * R + y) * (R / 64) + x / 64] |= 1ull << (x % 64); };
    set(17, 3, 10);
    set(0, 0, 0);
    set(63, 63, 63);
    vx_build* b = nullptr;
    vx::check(vx_build_dense(bits.data(), R, 6, &b));
    vx_scene_desc d{};
    vx::check(vx_build_desc(b, &d));
    vx::CudaOctree octree(d);
    vx_build_free(b);
    const struct { vx::Vec3 o, d; } rays[] = {
        {{-5.0f, 3.5f, 10.5f}, {1.0f, 0.0f, 0.0f}},
        {{17.5f, 40.0f, 10.5f}, {0.0f, -1.0f, 0.0f}},
        {{10.5f, 3.5f, 3.5f}, {1.0f, 0.0f, 1.0f}},
    };
    for (const auto& r : rays) {
        vx::RayHit h = octree.castRay(r.o, r.d, 0.0f, 1000.0f);
        std::printf("hit=%d t=%.6f pos=%d,%d,%d normal=%g,%g,%g scale=%d\n", int(h.hit), h.tMin, h.voxelPos[0],
                    h.voxelPos[1], h.voxelPos[2], h.normal.x, h.normal.y, h.normal.z, h.scale);
    }
    std::vector<vx_ray> batch(1000, vx_ray{17.5f, 40.0f, 10.5f, 0.0f, -1.0f, 0.0f});
    auto hits = octree.castRays(batch);
    int n = 0;
    for (const auto& h : hits) n += h.hit;
    std::printf("batch hits=%d\n", n);
    return 0;
}
