// vx_hash.h - Morton codes and the counter-based hash of the synthetic
// inputs, shared by the host builder and the device builder so that both
// produce the same brick order and the same payload bits.
#pragma once

#include <stdint.h>

#include "vx_hd.h"

namespace vx {

// 21-bit spread, x in bit 0 (MortonEncoding.cpp:19-27).
VX_HD uint64_t morton_expand3(uint32_t v) {
    uint64_t x = v & 0x1FFFFF;
    x = (x | x << 32) & 0x1F00000000FFFFULL;
    x = (x | x << 16) & 0x1F0000FF0000FFULL;
    x = (x | x << 8) & 0x100F00F00F00F00FULL;
    x = (x | x << 4) & 0x10C30C30C30C30C3ULL;
    x = (x | x << 2) & 0x1249249249249249ULL;
    return x;
}
VX_HD uint64_t morton3(uint32_t x, uint32_t y, uint32_t z) {
    return morton_expand3(x) | (morton_expand3(y) << 1) | (morton_expand3(z) << 2);
}
VX_HD uint32_t morton_compact3(uint64_t m) {
    m &= 0x1249249249249249ULL;
    m = (m ^ (m >> 2)) & 0x10C30C30C30C30C3ULL;
    m = (m ^ (m >> 4)) & 0x100F00F00F00F00FULL;
    m = (m ^ (m >> 8)) & 0x1F0000FF0000FFULL;
    m = (m ^ (m >> 16)) & 0x1F00000000FFFFULL;
    m = (m ^ (m >> 32)) & 0x1FFFFFULL;
    return uint32_t(m);
}

// Counter-based hash (seeded, deterministic).
VX_HD uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
VX_HD uint64_t hash4(uint64_t seed, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    uint64_t h = splitmix64(seed ^ 0x5851F42D4C957F2DULL);
    h = splitmix64(h ^ ((uint64_t(a) << 32) | b));
    h = splitmix64(h ^ ((uint64_t(c) << 32) | d));
    return h;
}

// Payload words of vx_synth_rgba8 / vx_synth_dxt1, keyed on the brick's grid
// coordinate (x | y << 10 | z << 20).
VX_HD uint32_t synth_rgba8_word(uint64_t seed, uint32_t coord, uint32_t voxel) {
    return uint32_t(hash4(seed, 0x72676261u, coord, voxel, 0)) | 0xFF000000u;
}
VX_HD uint64_t synth_dxt1_block(uint64_t seed, uint32_t coord, uint32_t block) {
    return hash4(seed, 0x64787431u, coord, block, 0);
}

}  // namespace vx
