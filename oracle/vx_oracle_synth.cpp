/*
 * vx_oracle_synth.cpp - the seeded synthetic inputs of the benchmark frames,
 * restated for the oracle side.
 *
 * TEST INFRASTRUCTURE ONLY (see vx_oracle.h).  The reference measures on
 * procedural scenes only, so the benchmark frames are seeded synthetic
 * scenes, cameras and secondary rays defined by this project.  The CPU
 * baseline and the reference arm of the benchmark build their inputs with
 * these functions so that they never load the product library; the CPU tests
 * check that they produce the product's bits (vx_synth_noise, vx_synth_urban,
 * vx_bounce_table, vx_spawn_bounce_rays, vx_spawn_shadow_rays).
 *
 * Definitions:
 *  - h(seed, a, b, c, d): splitmix64 chained over the seed and the packed
 *    words (a << 32 | b), (c << 32 | d).
 *  - value noise: octave o has lattice spacing s_o = spacing >> o and weight
 *    0.5^o; lattice value (h(seed, o, i, j, k) >> 40) * 2^-24; voxel centre
 *    p = (x + 0.5) / s_o; smoothstep weights w = f*f*(3 - 2f); blended along
 *    y, then z, then x; octaves summed in order.  Solid: value >= the value
 *    of ascending rank N - round(fill * N) (nothing solid when that count is
 *    0); a one-voxel box shell on request.
 *  - urban lattice: 32 x 32 blocks of pitch R / 32, streets max(1, R / 256)
 *    wide, block (bx, bz) a solid box of height min(R, hmin + h(seed,
 *    0x75726B, bx, bz, 0) mod (hmax - hmin + 1)).
 *  - bounce ray k of primary ray i: origin = o + normalize(d) * t moved 1e-3
 *    along the hit's face normal; direction = entry j = m(seed ^ m(2i + k))
 *    mod 4096 of a cosine-weighted table about +z (m = splitmix64), its z
 *    turned onto the normal's axis and sign.
 */
#include "vx_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

namespace {

uint64_t sm64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

uint64_t h4(uint64_t seed, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    uint64_t h = sm64(seed ^ 0x5851F42D4C957F2DULL);
    h = sm64(h ^ ((uint64_t(a) << 32) | b));
    return sm64(h ^ ((uint64_t(c) << 32) | d));
}

// Runs body(i) for i in [0, n) on `threads` threads (0: all cores), in
// interleaved blocks of 64 indices.
template <class F>
void for_each_index(int64_t n, int threads, F&& body) {
    int T = threads > 0 ? threads : int(std::max(1u, std::thread::hardware_concurrency()));
    T = int(std::min<int64_t>(T, std::max<int64_t>(1, n / 64)));
    std::atomic<int64_t> next{0};
    auto work = [&] {
        for (int64_t b; (b = next.fetch_add(64)) < n;)
            for (int64_t i = b; i < std::min(n, b + 64); ++i) body(i);
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < T; ++t) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
}

}  // namespace

extern "C" {

int vxo_synth_noise(uint32_t R, uint32_t spacing, uint32_t octaves, float fill, uint64_t seed, int32_t shell,
                    uint64_t* out, int threads) {
    if (!out || R < 64 || R % 64 || octaves < 1 || octaves > 16 || spacing < 1 || (spacing >> (octaves - 1)) < 1)
        return -1;
    const uint64_t N = uint64_t(R) * R * R;
    std::vector<float> value(N, 0.0f);
    for (uint32_t o = 0; o < octaves; ++o) {
        const uint32_t s = spacing >> o;
        const float fs = float(s);
        float weight = 1.0f;
        for (uint32_t k = 0; k < o; ++k) weight *= 0.5f;
        // lattice points along one axis: enough for every voxel centre and the +1 neighbour
        const uint32_t L = (R + s - 1) / s + 2;
        std::vector<float> lattice(size_t(L) * L * L);
        for_each_index(int64_t(L), threads, [&](int64_t k) {
            for (uint32_t j = 0; j < L; ++j)
                for (uint32_t i = 0; i < L; ++i)
                    lattice[(size_t(k) * L + j) * L + i] =
                        float(h4(seed, o, i, j, uint32_t(k)) >> 40) * (1.0f / 16777216.0f);
        });
        for_each_index(int64_t(R) * R, threads, [&](int64_t row) {
            const uint32_t y = uint32_t(row % R), z = uint32_t(row / R);
            const float py = (float(y) + 0.5f) / fs, pz = (float(z) + 0.5f) / fs;
            const float fy0 = std::floor(py), fz0 = std::floor(pz);
            const float fy = py - fy0, fz = pz - fz0;
            const float wy = fy * fy * (3.0f - 2.0f * fy), wz = fz * fz * (3.0f - 2.0f * fz);
            const uint32_t j = uint32_t(fy0), k = uint32_t(fz0);
            float* v = &value[size_t(row) * R];
            // the row's y-then-z blend at every lattice column it reaches, then one x blend per voxel
            const uint32_t cols = R / s + 2;
            std::vector<float> yz(cols);
            const float* l = lattice.data();
            for (uint32_t i = 0; i < cols; ++i) {
                const float c00 = l[(size_t(k) * L + j) * L + i];
                const float c10 = l[(size_t(k) * L + j + 1) * L + i];
                const float c01 = l[(size_t(k + 1) * L + j) * L + i];
                const float c11 = l[(size_t(k + 1) * L + j + 1) * L + i];
                const float alongY0 = c00 + wy * (c10 - c00);
                const float alongY1 = c01 + wy * (c11 - c01);
                yz[i] = alongY0 + wz * (alongY1 - alongY0);
            }
            for (uint32_t x = 0; x < R; ++x) {
                const float px = (float(x) + 0.5f) / fs;
                const float fx0 = std::floor(px);
                const float fx = px - fx0;
                const float wx = fx * fx * (3.0f - 2.0f * fx);
                const uint32_t i = uint32_t(fx0);
                v[x] = v[x] + weight * (yz[i] + wx * (yz[i + 1] - yz[i]));
            }
        });
    }
    // Threshold: the value of ascending rank N - n_solid.  The values are
    // non-negative, so their bit patterns order like the values: find the
    // pattern's top 16 bits from one histogram, then its low 16 bits from a
    // second histogram over the values with those top bits.
    const uint64_t n_solid = uint64_t(std::floor(double(fill) * double(N) + 0.5));
    uint32_t thr = 0xFFFFFFFFu;
    if (n_solid > 0) {
        uint64_t rank = N - n_solid;
        auto histogram = [&](bool low, uint32_t top) {
            const int T = threads > 0 ? threads : int(std::max(1u, std::thread::hardware_concurrency()));
            std::vector<std::vector<uint64_t>> part(size_t(T), std::vector<uint64_t>(65536, 0));
            std::vector<std::thread> pool;
            for (int t = 0; t < T; ++t)
                pool.emplace_back([&, t] {
                    std::vector<uint64_t>& hst = part[size_t(t)];
                    const uint64_t b = N * uint64_t(t) / T, e = N * uint64_t(t + 1) / T;
                    for (uint64_t q = b; q < e; ++q) {
                        uint32_t u;
                        std::memcpy(&u, &value[q], 4);
                        if (!low) hst[u >> 16]++;
                        else if ((u >> 16) == top) hst[u & 0xFFFFu]++;
                    }
                });
            for (auto& th : pool) th.join();
            std::vector<uint64_t> sum(65536, 0);
            for (const auto& p : part)
                for (size_t i = 0; i < 65536; ++i) sum[i] += p[i];
            return sum;
        };
        auto pick = [&](const std::vector<uint64_t>& hst) {
            for (uint32_t b = 0; b < 65536; ++b) {
                if (rank < hst[b]) return b;
                rank -= hst[b];
            }
            return 65535u;
        };
        const uint32_t top = pick(histogram(false, 0));
        const uint32_t bottom = pick(histogram(true, top));
        thr = (top << 16) | bottom;
    }
    float t;
    std::memcpy(&t, &thr, 4);
    const uint32_t wpr = R / 64;
    for_each_index(int64_t(R) * R, threads, [&](int64_t row) {
        const uint32_t y = uint32_t(row % R), z = uint32_t(row / R);
        const float* v = &value[size_t(row) * R];
        const bool edge_row = y == 0 || z == 0 || y == R - 1 || z == R - 1;
        for (uint32_t w = 0; w < wpr; ++w) {
            uint64_t bitsw = 0;
            for (uint32_t b = 0; b < 64; ++b) {
                const uint32_t x = w * 64 + b;
                bool solid = n_solid > 0 && v[x] >= t;
                if (shell && (edge_row || x == 0 || x == R - 1)) solid = true;
                if (solid) bitsw |= uint64_t(1) << b;
            }
            out[size_t(row) * wpr + w] = bitsw;
        }
    });
    return 0;
}

int vxo_synth_urban(uint32_t R, uint32_t hmin, uint32_t hmax, uint64_t seed, uint64_t* out) {
    if (!out || R < 64 || R % 64 || hmin > hmax) return -1;
    const uint32_t pitch = R / 32, street = std::max(1u, R / 256), wpr = R / 64;
    uint32_t top[32][32];
    for (uint32_t bz = 0; bz < 32; ++bz)
        for (uint32_t bx = 0; bx < 32; ++bx)
            top[bz][bx] = std::min(R, hmin + uint32_t(h4(seed, 0x75726Bu, bx, bz, 0) % uint64_t(hmax - hmin + 1)));
    for_each_index(int64_t(R) * R, 0, [&](int64_t row) {
        const uint32_t y = uint32_t(row % R), z = uint32_t(row / R);
        const bool in_z = (z % pitch) < pitch - street;
        for (uint32_t w = 0; w < wpr; ++w) {
            uint64_t bitsw = 0;
            for (uint32_t b = 0; b < 64; ++b) {
                const uint32_t x = w * 64 + b;
                if (in_z && (x % pitch) < pitch - street && y < top[z / pitch][x / pitch]) bitsw |= uint64_t(1) << b;
            }
            out[size_t(row) * wpr + w] = bitsw;
        }
    });
    return 0;
}

// Material colours.  vxo_material_color_cpu: MaterialIdToColor
// (SVO/src/SVORebuild.cpp:68-120), the colour the compressed payload is
// encoded from.  vxo_material_color_shader: getMaterialColor
// (shaders/Materials.glsl:18-60) of the uncompressed compute shader, whose
// ids 33-39 are mix(stone0, stone1, (id - 33) / 6) with GLSL's
// mix(x, y, a) = x * (1 - a) + y * a.  Both end in the same HSV wheel.
namespace {
struct Entry { uint32_t id; float r, g, b; };
const Entry kListed[] = {
    {1, 1.0f, 0.0f, 0.0f},     {2, 0.0f, 1.0f, 0.0f},     {3, 0.9f, 0.9f, 0.9f},     {4, 0.85f, 0.85f, 0.85f},
    {5, 0.95f, 0.95f, 0.95f},  {6, 0.8f, 0.8f, 0.8f},     {7, 0.4f, 0.4f, 0.4f},     {10, 0.8f, 0.6f, 0.2f},
    {11, 0.6f, 0.8f, 0.9f},    {20, 1.0f, 0.98f, 0.9f},   {30, 0.5f, 0.45f, 0.4f},   {31, 0.6f, 0.55f, 0.5f},
    {32, 0.55f, 0.5f, 0.45f},  {40, 0.8f, 0.6f, 0.2f},    {50, 0.2f, 0.2f, 0.22f},   {60, 0.6f, 0.58f, 0.55f},
    {61, 0.7f, 0.85f, 0.95f}};
const Entry kStoneCpu[] = {
    {33, 0.52f, 0.48f, 0.42f}, {34, 0.48f, 0.44f, 0.38f}, {35, 0.45f, 0.42f, 0.36f}, {36, 0.58f, 0.52f, 0.46f},
    {37, 0.62f, 0.56f, 0.48f}, {38, 0.65f, 0.58f, 0.5f},  {39, 0.68f, 0.6f, 0.52f}};

bool lookup(const Entry* t, size_t n, uint32_t id, float out[3]) {
    for (size_t k = 0; k < n; ++k)
        if (t[k].id == id) {
            out[0] = t[k].r; out[1] = t[k].g; out[2] = t[k].b;
            return true;
        }
    return false;
}

void hsv_wheel(uint32_t id, float out[3]) {
    const float hue = static_cast<float>(id % 256) / 256.0f;
    const float h = hue * 6.0f;
    const int i = static_cast<int>(h);
    const float f = h - static_cast<float>(i);
    const float p = 0.8f * 0.3f, q = 0.8f * (1.0f - 0.7f * f), t = 0.8f * (1.0f - 0.7f * (1.0f - f));
    const float rows[6][3] = {{0.8f, t, p}, {q, 0.8f, p}, {p, 0.8f, t}, {p, q, 0.8f}, {t, p, 0.8f}, {0.8f, p, q}};
    const int r = i < 5 ? i : 5;
    out[0] = rows[r][0]; out[1] = rows[r][1]; out[2] = rows[r][2];
}
}  // namespace

void vxo_material_color_cpu(uint32_t id, float out[3]) {
    if (lookup(kListed, sizeof(kListed) / sizeof(kListed[0]), id, out)) return;
    if (lookup(kStoneCpu, sizeof(kStoneCpu) / sizeof(kStoneCpu[0]), id, out)) return;
    hsv_wheel(id, out);
}

void vxo_material_color_shader(uint32_t id, float out[3]) {
    if (lookup(kListed, sizeof(kListed) / sizeof(kListed[0]), id, out)) return;
    if (id >= 33 && id <= 39) {
        const float a = static_cast<float>(id - 33) / 6.0f;
        const float lo[3] = {0.52f, 0.48f, 0.42f}, hi[3] = {0.68f, 0.6f, 0.52f};
        for (int c = 0; c < 3; ++c) out[c] = lo[c] * (1.0f - a) + hi[c] * a;
        return;
    }
    hsv_wheel(id, out);
}

void vxo_bounce_table(float* out) {
    for (uint32_t k = 0; k < 4096; ++k) {
        const uint64_t a = sm64(0xB0C0E5EEDULL + k), b = sm64(a);
        const double u1 = double(a >> 11) / 9007199254740992.0;
        const double u2 = double(b >> 11) / 9007199254740992.0;
        const double radius = std::sqrt(u1), angle = 6.283185307179586476925 * u2;
        out[3 * k] = float(radius * std::cos(angle));
        out[3 * k + 1] = float(radius * std::sin(angle));
        out[3 * k + 2] = float(std::sqrt(std::max(0.0, 1.0 - u1)));
    }
}

// Secondary rays from the oracle's hit records.  kind 0: two bounce rays per
// primary ray (out: 2n rays); kind 1: one shadow ray toward light (out: n).
// index[i] (NULL: i) is ray i's position in its frame, which picks its bounce
// directions.  Misses give rays with the primary origin and a zero direction.
void vxo_spawn_rays(const float* rays, const vxo_hit* hits, const uint64_t* index, uint64_t n, int kind,
                    uint64_t seed, const float light[3], float* out) {
    static const std::vector<float> table = [] {
        std::vector<float> t(4096 * 3);
        vxo_bounce_table(t.data());
        return t;
    }();
    const int per = kind == 0 ? 2 : 1;
    for (uint64_t i = 0; i < n; ++i) {
        const float* r = rays + 6 * i;
        float* o = out + 6 * per * i;
        const bool hit = hits[i].flags & 1u;
        float org[3] = {r[0], r[1], r[2]};
        int axis = 0;
        float sgn = 1.0f;
        if (hit) {
            const float len2 = (r[3] * r[3] + r[4] * r[4]) + r[5] * r[5];
            const float inv = 1.0f / std::sqrt(len2);
            for (int a = 0; a < 3; ++a) org[a] = r[a] + (r[3 + a] * inv) * hits[i].t;
            axis = int((hits[i].flags >> 1) & 3u);
            sgn = (hits[i].flags & 8u) ? -1.0f : 1.0f;
            org[axis] = org[axis] + sgn * 0.001f;
        }
        for (int k = 0; k < per; ++k) {
            float* q = o + 6 * k;
            q[0] = org[0]; q[1] = org[1]; q[2] = org[2];
            q[3] = q[4] = q[5] = 0.0f;
            if (!hit) continue;
            if (kind == 1) {
                q[3] = light[0]; q[4] = light[1]; q[5] = light[2];
                continue;
            }
            const uint64_t fi = index ? index[i] : i;
            const uint32_t j = uint32_t(sm64(seed ^ sm64((fi << 1) | uint64_t(k))) & 4095u);
            const float tu = table[3 * j], tv = table[3 * j + 1], tw = table[3 * j + 2] * sgn;
            // the table's +z onto the normal axis: x-normal (w, u, v), y-normal (v, w, u), z-normal (u, v, w)
            const float d[3][3] = {{tw, tu, tv}, {tv, tw, tu}, {tu, tv, tw}};
            q[3] = d[axis][0]; q[4] = d[axis][1]; q[5] = d[axis][2];
        }
    }
}

}  // extern "C"
