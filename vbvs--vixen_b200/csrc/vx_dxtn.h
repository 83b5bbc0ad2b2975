// vx_dxtn.h - DXT normal blocks, shared by the host builder, the GPU builder
// and the shading kernels (host and device compile the same IEEE binary32
// operation sequence: no contraction, IEEE division and square root).
//
// Block format (DXTNormalBlock, VoxelData/include/Compression/DXT1Compressor.h;
// addressing VoxelRayMarch_Compressed.comp:142-150): 16 B per 16 consecutive
// brick voxels, {blockA = headBase | bitsU << 32, blockB = headUV | bitsV << 32}.
//   headBase  base normal: sign of the dominant component (bit 31), dominant
//             axis (bits 29-30), the two others as 15- and 14-bit ratios
//   headUV    two axis vectors U (bits 0-15) and V (bits 16-31): a 4-bit
//             exponent and three 4-bit offset-binary components each
//   bitsU/V   2-bit weights per texel from {-1, -1/3, 1/3, 1}
// Decoded texel = (base + U * wU) + V * wV (DXTNormalCompressor::decodeBlockTyped,
// DXT1Compressor.cpp:335-354; decodeDXTNormal, shaders/Compression.glsl:158-177).
//
// The encoder is DXTNormalCompressor::encodeBlockTyped (DXT1Compressor.cpp:242-333)
// and the per-voxel input is the rebuild's geometric normal
// (computeGeometricNormal, SVO/src/SVORebuild.cpp:145-193): both must produce the
// reference's bits, so their steps are the reference's.
#pragma once

#include <stdint.h>
#include <string.h>

#include <cmath>

#include "vx_hd.h"

namespace vx {
namespace dxtn {

struct F3 {
    float x, y, z;
};

VX_HD F3 f3(float x, float y, float z) { return F3{x, y, z}; }
VX_HD F3 operator+(F3 a, F3 b) { return F3{a.x + b.x, a.y + b.y, a.z + b.z}; }
VX_HD F3 operator-(F3 a, F3 b) { return F3{a.x - b.x, a.y - b.y, a.z - b.z}; }
VX_HD F3 operator*(F3 a, float s) { return F3{a.x * s, a.y * s, a.z * s}; }
// glm::dot: (x*x' + y*y') + z*z'
VX_HD float dot(F3 a, F3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
VX_HD float len(F3 a) { return sqrtf(dot(a, a)); }
// glm::normalize: v * (1 / sqrt(dot(v, v)))
VX_HD F3 unit(F3 a) { return a * (1.0f / sqrtf(dot(a, a))); }

// 2^e for e in [-126, 127], exact.
VX_HD float pow2(int e) {
    const uint32_t b = uint32_t(e + 127) << 23;
    float f;
    memcpy(&f, &b, 4);
    return f;
}
VX_HD uint32_t fbits(float f) {
    uint32_t b;
    memcpy(&b, &f, 4);
    return b;
}
// static_cast<int>(float) as x86-64 evaluates it (INT_MIN out of range).
VX_HD int trunc_i(float f) { return (f >= -2147483648.0f && f < 2147483648.0f) ? int(f) : int(0x80000000u); }
VX_HD int clampi(int v, int lo, int hi) { return v < lo ? lo : (hi < v ? hi : v); }
VX_HD float absf(float v) { return fabsf(v); }

// {-1, -1/3, 1/3, 1}
VX_HD float weight(uint32_t sel) {
    return sel == 0 ? -1.0f : sel == 1 ? (-1.0f / 3.0f) : sel == 2 ? (1.0f / 3.0f) : 1.0f;
}

// encodeRawNormal (DXT1Compressor.cpp:168-193)
VX_HD uint32_t pack_base(F3 n) {
    const float ax = absf(n.x), ay = absf(n.y), az = absf(n.z);
    const float yz = (ay < az) ? az : ay;
    const int axis = (ax >= yz) ? 0 : (ay >= az) ? 1 : 2;
    const float t = axis == 0 ? n.x : axis == 1 ? n.y : n.z;
    const float u = axis == 0 ? n.y : axis == 1 ? n.z : n.x;
    const float v = axis == 0 ? n.z : axis == 1 ? n.x : n.y;
    uint32_t r = (t < 0.0f ? 0x80000000u : 0u) | (uint32_t(axis) << 29);
    const float at = absf(t);
    if (at > 0.0f) {
        const int iu = clampi(trunc_i((u / at) * 16383.0f), -0x4000, 0x3FFF);
        const int iv = clampi(trunc_i((v / at) * 8191.0f), -0x2000, 0x1FFF);
        r |= (uint32_t(iu) & 0x7FFFu) << 14;
        r |= uint32_t(iv) & 0x3FFFu;
    }
    return r;
}

// decodeRawNormal (:195-207)
VX_HD F3 unpack_base(uint32_t w) {
    const int32_t t = (int32_t(w) >> 31) ^ 0x7FFFFFFF;
    const int32_t u = int32_t(w << 3);
    const int32_t v = int32_t(w << 18);
    const uint32_t axis = (w >> 29) & 3u;
    if (axis == 0) return F3{float(t), float(u), float(v)};
    if (axis == 1) return F3{float(v), float(t), float(u)};
    return F3{float(u), float(v), float(t)};
}

// encodeNormalAxis (:209-228): the exponent of the largest component, then the
// z, y, x nibbles, each rounded against the bits already written.
VX_HD uint32_t pack_axis(uint32_t head, F3 a, int shift) {
    float m = absf(a.x);
    if (m < absf(a.y)) m = absf(a.y);
    if (m < absf(a.z)) m = absf(a.z);
    int e = 0;
    if (m > 0.0f) e = clampi(int(fbits(m) >> 23) + (-127 - 31 + 1 - 3 + 13), 0, 15);
    const F3 s = a * pow2(-e + (13 - 31));
    head |= uint32_t(e) << shift;
    head |= uint32_t(clampi(trunc_i((s.z + 8.5f) - float(head) * pow2(-4 - shift)), 0, 15) ^ 8) << (4 + shift);
    head |= uint32_t(clampi(trunc_i((s.y + 8.5f) - float(head) * pow2(-8 - shift)), 0, 15) ^ 8) << (8 + shift);
    head |= uint32_t(clampi(trunc_i((s.x + 8.5f) - float(head) * pow2(-12 - shift)), 0, 15) ^ 8) << (12 + shift);
    return head;
}

// decodeNormalAxis (:230-240)
VX_HD F3 unpack_axis(uint32_t head, int shift) {
    const int32_t sh = int32_t(head << (16 - shift));
    const float sc = pow2(((sh >> 16) & 15) + (3 - 13));
    return F3{float(sh) * sc, float(int32_t(uint32_t(sh) << 4)) * sc, float(int32_t(uint32_t(sh) << 8)) * sc};
}

// Unnormalised texel t of a block.
VX_HD F3 decode(uint64_t a, uint64_t b, uint32_t t) {
    const F3 base = unpack_base(uint32_t(a));
    const F3 u = unpack_axis(uint32_t(b), 0);
    const F3 v = unpack_axis(uint32_t(b), 16);
    const float wu = weight((uint32_t(a >> 32) >> (2u * t)) & 3u);
    const float wv = weight((uint32_t(b >> 32) >> (2u * t)) & 3u);
    return (base + u * wu) + v * wv;
}

// encodeBlockTyped over all 16 texels (the rebuild passes validCount = 16).
VX_HD void encode(const F3* n, uint64_t& out_a, uint64_t& out_b) {
    F3 base = n[0];
    for (int i = 1; i < 16; ++i) base = base + n[i];
    if (len(base) < 0.1f * 16.0f) {
        // nearly cancelling normals: the input closest to the sum
        int bi = 0;
        float bd = dot(n[0], base);
        for (int i = 1; i < 16; ++i) {
            const float d = dot(n[i], base);
            if (d > bd) { bi = i; bd = d; }
        }
        base = n[bi];
    }
    const uint32_t head_base = pack_base(base);
    base = unpack_base(head_base);
    // U: toward the input furthest from the base
    int ui = 0;
    float ud = dot(n[0], base);
    for (int i = 1; i < 16; ++i) {
        const float d = dot(n[i], base);
        if (d < ud) { ui = i; ud = d; }
    }
    uint32_t head_uv = pack_axis(0u, n[ui] * len(base) - base, 0);
    const F3 u = unpack_axis(head_uv, 0);
    // V: toward the input the U line fits worst
    F3 uref[4];
    for (int j = 0; j < 4; ++j) uref[j] = unit(base + u * weight(uint32_t(j)));
    int vi = 0, vj = 0;
    float vd = 3.402823466e+38f;
    for (int i = 0; i < 16; ++i) {
        int bj = 0;
        float bd = dot(n[i], uref[0]);
        for (int j = 1; j < 4; ++j) {
            const float d = dot(n[i], uref[j]);
            if (d > bd) { bj = j; bd = d; }
        }
        if (bd < vd) { vi = i; vj = bj; vd = bd; }
    }
    const F3 tmp = base + u * weight(uint32_t(vj));
    head_uv = pack_axis(head_uv, n[vi] * len(tmp) - tmp, 16);
    const F3 v = unpack_axis(head_uv, 16);
    // weights: the best of the 4 x 4 grid per texel
    F3 grid[16];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) grid[i + 4 * j] = unit((base + u * weight(uint32_t(i))) + v * weight(uint32_t(j)));
    uint32_t bu = 0, bv = 0;
    for (int t = 0; t < 16; ++t) {
        int bk = 0;
        float bd = dot(n[t], grid[0]);
        for (int k = 1; k < 16; ++k) {
            const float d = dot(n[t], grid[k]);
            if (d > bd) { bk = k; bd = d; }
        }
        bu |= uint32_t(bk & 3) << (2 * t);
        bv |= uint32_t(bk >> 2) << (2 * t);
    }
    out_a = uint64_t(head_base) | (uint64_t(bu) << 32);
    out_b = uint64_t(head_uv) | (uint64_t(bv) << 32);
}

VX_HD bool occupied(const uint32_t* occ, int x, int y, int z) {
    if (unsigned(x) > 7u || unsigned(y) > 7u || unsigned(z) > 7u) return false;
    const int i = z * 64 + y * 8 + x;
    return (occ[i >> 5] >> (i & 31)) & 1u;
}

// computeGeometricNormal: outward central difference of the brick's
// occupancy (neighbours outside the brick count as empty); (0,1,0) when flat.
VX_HD F3 geometric(const uint32_t* occ, int x, int y, int z) {
    auto o = [&](int X, int Y, int Z) { return occupied(occ, X, Y, Z) ? 1.0f : 0.0f; };
    const F3 g{o(x + 1, y, z) - o(x - 1, y, z), o(x, y + 1, z) - o(x, y - 1, z), o(x, y, z + 1) - o(x, y, z - 1)};
    if (len(g) > 0.001f) {
        const F3 u = unit(g);
        return F3{-u.x, -u.y, -u.z};
    }
    return F3{0.0f, 1.0f, 0.0f};
}

// One block of a brick's normal payload (SVORebuild.cpp:658-722): empty texels
// are (0,1,0); a block without occupied texels is {0, 0}.
VX_HD void brick_block(const uint32_t* occ, int block, uint64_t& a, uint64_t& b) {
    F3 n[16];
    bool any = false;
    for (int t = 0; t < 16; ++t) {
        const int i = block * 16 + t;
        const int x = i & 7, y = (i >> 3) & 7, z = i >> 6;
        const bool occd = occupied(occ, x, y, z);
        any = any || occd;
        n[t] = occd ? geometric(occ, x, y, z) : F3{0.0f, 1.0f, 0.0f};
    }
    if (any) encode(n, a, b);
    else a = b = 0;
}

}  // namespace dxtn
}  // namespace vx
