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

// computeGeometricNormal (SVO/src/SVORebuild.cpp:145-193) takes the central
// difference g of the brick's occupancy (neighbours outside the brick count as
// empty) and returns the outward unit normal -normalize(g), or (0,1,0) when g
// is (near) zero.
VX_HD F3 normal_of_gradient(F3 g) {
    if (len(g) > 0.001f) {
        const F3 u = unit(g);
        return F3{-u.x, -u.y, -u.z};
    }
    return F3{0.0f, 1.0f, 0.0f};
}

// The encoder's input normal of a texel is a function of its neighbour code
// c = (gx + 1) + 3 (gy + 1) + 9 (gz + 1) alone, g in {-1, 0, 1}^3 the central
// difference: the reference forms each component of g as a difference of
// occupancy floats, 1 - 0, 0 - 1, 0 - 0 or 1 - 1, i.e. exactly float(gx) etc.
// (+0 for the zero cases), so code_normal(c) returns the bits of that texel's
// normal.  Empty texels take FLAT_CODE: g = 0 gives (0,1,0), the empty texel's
// normal, bit for bit.
constexpr int NUM_CODES = 27;
constexpr int FLAT_CODE = 13;

VX_HD F3 code_normal(int c) {
    return normal_of_gradient(F3{float(c % 3 - 1), float(c / 3 % 3 - 1), float(c / 9 - 1)});
}

// code_normal of every code, as 16-byte entries {x, y, z, 0} (shared memory on
// the device: one 128-bit load per lookup).
struct CodeTable {
    const float4* e;
    VX_HD F3 operator()(int c) const {
        const float4 q = e[c];
        return F3{q.x, q.y, q.z};
    }
};

VX_HD float4 code_entry(int c) {
    const F3 n = code_normal(c);
    return float4{n.x, n.y, n.z, 0.0f};
}

// Occupancy row (8 bits, x = bit) of row y of slice z; 0 outside the brick.
VX_HD uint32_t row8(const uint32_t* occ, int y, int z) {
    if (unsigned(y) > 7u || unsigned(z) > 7u) return 0u;
    return (occ[2 * z + (y >> 2)] >> ((y & 3) * 8)) & 0xFFu;
}

// Neighbour codes of the 16 texels of block `block` (voxels block*16 ..
// block*16 + 15: rows y = 2p and 2p + 1 of slice z, p = block & 3,
// z = block >> 2).  Returns whether any texel is occupied.
VX_HD bool block_codes(const uint32_t* occ, int block, uint8_t* code) {
    const int z = block >> 2, y0 = (block & 3) * 2;
    bool any = false;
    VX_UNROLL
    for (int r = 0; r < 2; ++r) {
        const int y = y0 + r;
        const uint32_t row = row8(occ, y, z);
        any = any || row != 0u;
        const uint32_t xp = row >> 1, xm = (row << 1) & 0xFFu;
        const uint32_t yp = row8(occ, y + 1, z), ym = row8(occ, y - 1, z);
        const uint32_t zp = row8(occ, y, z + 1), zm = row8(occ, y, z - 1);
        VX_UNROLL
        for (int x = 0; x < 8; ++x) {
            const int c = FLAT_CODE + (int((xp >> x) & 1u) - int((xm >> x) & 1u)) +
                          3 * (int((yp >> x) & 1u) - int((ym >> x) & 1u)) +
                          9 * (int((zp >> x) & 1u) - int((zm >> x) & 1u));
            code[r * 8 + x] = uint8_t(((row >> x) & 1u) ? c : FLAT_CODE);
        }
    }
    return any;
}

// encodeBlockTyped (DXT1Compressor.cpp:242-333) over all 16 texels (the rebuild
// passes validCount = 16), for texels given as neighbour codes.  Every step is
// the reference's over the 16 texel normals in order, except that the searches
// visit each distinct normal once, in the order of first occurrence.  That is
// exact: a later texel with the same normal yields the same value, and a value
// equal to one already seen never passes a strict comparison whose running best
// is at least as good (or NaN, which blocks all), so the reference's pick is
// always a first occurrence.  The distinct codes sit in a byte list (two
// 64-bit words), so the searches run `m` iterations, m the number of distinct
// normals of the block, instead of 16.
VX_HD void encode_coded(const uint8_t* code, CodeTable tab, uint64_t& out_a, uint64_t& out_b) {
    uint64_t list0 = 0, list1 = 0;  // distinct codes, first occurrences in texel order
    uint32_t seen = 0;
    int m = 0;
    VX_UNROLL
    for (int t = 0; t < 16; ++t) {
        const uint32_t bit = 1u << code[t];
        if (!(seen & bit)) {
            const uint64_t e = uint64_t(code[t]) << (8 * (m & 7));
            if (m < 8) list0 |= e;
            else list1 |= e;
            ++m;
        }
        seen |= bit;
    }
    const auto listed = [&](int j) { return int(((j < 8 ? list0 : list1) >> (8 * (j & 7))) & 0xFFu); };
    F3 base = tab(code[0]);
    VX_UNROLL
    for (int t = 1; t < 16; ++t) base = base + tab(code[t]);
    if (len(base) < 0.1f * 16.0f) {
        // nearly cancelling normals: the input closest to the sum
        int bc = code[0];
        float bd = dot(tab(code[0]), base);
        for (int j = 1; j < m; ++j) {
            const int c = listed(j);
            const float d = dot(tab(c), base);
            if (d > bd) { bc = c; bd = d; }
        }
        base = tab(bc);
    }
    const uint32_t head_base = pack_base(base);
    base = unpack_base(head_base);
    // U: toward the input furthest from the base
    int uc = code[0];
    float ud = dot(tab(code[0]), base);
    for (int j = 1; j < m; ++j) {
        const int c = listed(j);
        const float d = dot(tab(c), base);
        if (d < ud) { uc = c; ud = d; }
    }
    uint32_t head_uv = pack_axis(0u, tab(uc) * len(base) - base, 0);
    const F3 u = unpack_axis(head_uv, 0);
    // V: toward the input the U line fits worst
    F3 uref[4];
    VX_UNROLL
    for (int j = 0; j < 4; ++j) uref[j] = unit(base + u * weight(uint32_t(j)));
    int vc = code[0], vj = 0;
    float vd = 3.402823466e+38f;
    for (int j = 0; j < m; ++j) {
        const int c = listed(j);
        const F3 n = tab(c);
        int bj = 0;
        float bd = dot(n, uref[0]);
        VX_UNROLL
        for (int i = 1; i < 4; ++i) {
            const float d = dot(n, uref[i]);
            if (d > bd) { bj = i; bd = d; }
        }
        if (bd < vd) { vc = c; vj = bj; vd = bd; }
    }
    const F3 tmp = base + u * weight(uint32_t(vj));
    head_uv = pack_axis(head_uv, tab(vc) * len(tmp) - tmp, 16);
    const F3 v = unpack_axis(head_uv, 16);
    // weights: the best of the 4 x 4 grid, once per distinct normal, kept per code
    F3 grid[16];
    VX_UNROLL
    for (int i = 0; i < 4; ++i)
        VX_UNROLL
        for (int j = 0; j < 4; ++j) grid[i + 4 * j] = unit((base + u * weight(uint32_t(i))) + v * weight(uint32_t(j)));
    uint64_t best_lo = 0, best_hi = 0;  // 4 bits per code: codes 0-15, 16-26
    for (int j = 0; j < m; ++j) {
        const int c = listed(j);
        const F3 n = tab(c);
        int bk = 0;
        float bd = dot(n, grid[0]);
        VX_UNROLL
        for (int k = 1; k < 16; ++k) {
            const float d = dot(n, grid[k]);
            if (d > bd) { bk = k; bd = d; }
        }
        if (c < 16) best_lo |= uint64_t(bk) << (4 * c);
        else best_hi |= uint64_t(bk) << (4 * (c - 16));
    }
    uint32_t bu = 0, bv = 0;
    VX_UNROLL
    for (int t = 0; t < 16; ++t) {
        const int c = code[t];
        const uint32_t bk = uint32_t(c < 16 ? best_lo >> (4 * c) : best_hi >> (4 * (c - 16))) & 15u;
        bu |= (bk & 3u) << (2 * t);
        bv |= (bk >> 2) << (2 * t);
    }
    out_a = uint64_t(head_base) | (uint64_t(bu) << 32);
    out_b = uint64_t(head_uv) | (uint64_t(bv) << 32);
}

// One block of a brick's normal payload (SVORebuild.cpp:658-722): empty texels
// are (0,1,0); a block without occupied texels is {0, 0}.
VX_HD void brick_block(const uint32_t* occ, int block, CodeTable tab, uint64_t& a, uint64_t& b) {
    uint8_t code[16];
    if (block_codes(occ, block, code)) encode_coded(code, tab, a, b);
    else a = b = 0;
}

}  // namespace dxtn
}  // namespace vx
