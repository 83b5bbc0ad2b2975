// vx_dxt1.h - DXT1 colour blocks (DXT1ColorCompressor,
// VoxelData/src/Compression/DXT1Compressor.cpp:14-111), shared by the host and
// device payload builders.  Block: head = two RGB-565 endpoints (ref0 in bits
// 0-15, ref1 in 16-31, blue lowest), bits = 2-bit selectors of 16 texels;
// ref2 = 2/3 ref0 + 1/3 ref1, ref3 = 1/3 ref0 + 2/3 ref1.  The encoder must
// produce the reference's bits, so its steps are the reference's:
// endpoints = the farthest pair of inputs, residual-corrected 565 rounding,
// each texel the nearest of the four decoded references.
#pragma once

#include <stdint.h>

#include "vx_hd.h"

namespace vx {
namespace dxt1 {

struct C3 {
    float r, g, b;
};

VX_HD float dist2(C3 a, C3 b) {
    const float x = a.r - b.r, y = a.g - b.g, z = a.b - b.b;
    return (x * x + y * y) + z * z;
}
VX_HD int trunc_i(float f) { return (f >= -2147483648.0f && f < 2147483648.0f) ? int(f) : int(0x80000000u); }
VX_HD uint32_t quant(float v, float m, float sub, int hi) {
    const int q = trunc_i((v * m + 0.5f) - sub);
    return uint32_t(q < 0 ? 0 : (hi < q ? hi : q));
}

// encodeColorHead (:38-55); the exp2 factors are exact powers of two.
VX_HD uint32_t encode_head(C3 c0, C3 c1) {
    uint32_t h = quant(c0.b, 31.0f, 0.0f, 31);
    h |= quant(c0.g, 63.0f, float(h) * (1.0f / 32.0f), 63) << 5;
    h |= quant(c0.r, 31.0f, float(h) * (1.0f / 2048.0f), 31) << 11;
    h |= quant(c1.b, 31.0f, float(h) * (1.0f / 65536.0f), 31) << 16;
    h |= quant(c1.g, 63.0f, float(h) * (1.0f / 2097152.0f), 63) << 21;
    h |= quant(c1.r, 31.0f, float(h) * (1.0f / 134217728.0f), 31) << 27;
    return h;
}

// decodeColorHead (:14-36)
VX_HD void decode_head(uint32_t head, C3 ref[4]) {
    const float s = 1.0f / 4294967296.0f;
    ref[0] = C3{float(head << 16) * s, float(head << 21) * s, float(head << 27) * s};
    ref[1] = C3{float(head) * s, float(head << 5) * s, float(head << 11) * s};
    ref[2] = C3{ref[0].r * (2.0f / 3.0f) + ref[1].r * (1.0f / 3.0f), ref[0].g * (2.0f / 3.0f) + ref[1].g * (1.0f / 3.0f),
                ref[0].b * (2.0f / 3.0f) + ref[1].b * (1.0f / 3.0f)};
    ref[3] = C3{ref[0].r * (1.0f / 3.0f) + ref[1].r * (2.0f / 3.0f), ref[0].g * (1.0f / 3.0f) + ref[1].g * (2.0f / 3.0f),
                ref[0].b * (1.0f / 3.0f) + ref[1].b * (2.0f / 3.0f)};
}

VX_HD C3 texel(const float* p, int t) { return C3{p[3 * t], p[3 * t + 1], p[3 * t + 2]}; }

// encodeBlockTyped (:57-111) over 16 texels, texel t at p[3t .. 3t + 2].
VX_HD uint64_t encode16(const float* p) {
    int i0 = 0, i1 = 0;
    float best = -3.402823466e+38f;
    VX_UNROLL
    for (int i = 0; i < 16; ++i)
        VX_UNROLL
        for (int j = i + 1; j < 16; ++j) {
            const float d = dist2(texel(p, i), texel(p, j));
            if (d > best) { i0 = i; i1 = j; best = d; }
        }
    const uint32_t head = encode_head(texel(p, i0), texel(p, i1));
    C3 ref[4];
    decode_head(head, ref);
    uint32_t bits = 0;
    VX_UNROLL
    for (int t = 0; t < 16; ++t) {
        const C3 c = texel(p, t);
        int bi = 0;
        float bd = 3.402823466e+38f;
        VX_UNROLL
        for (int j = 0; j < 4; ++j) {
            const float d = dist2(c, ref[j]);
            if (d < bd) { bi = j; bd = d; }
        }
        bits |= uint32_t(bi) << (2 * t);
    }
    return uint64_t(head) | (uint64_t(bits) << 32);
}

// Zero the empty texels of a 16-texel block in place (the rebuild's input for
// them is (0,0,0)).
VX_HD void mask_empty(float* p, uint32_t occ16) {
    VX_UNROLL
    for (int t = 0; t < 16; ++t)
        if (!((occ16 >> t) & 1u)) p[3 * t] = p[3 * t + 1] = p[3 * t + 2] = 0.0f;
}

// Block k of a brick's colour payload (SVORebuild.cpp:658-722); rgb: the
// brick's 512 x 3 floats, occ its 16 occupancy words.  A block without
// occupied texels is 0.
VX_HD uint64_t brick_block(const float* rgb, const uint32_t* occ, int k) {
    const uint32_t occ16 = (occ[k >> 1] >> ((k & 1) * 16)) & 0xFFFFu;
    if (!occ16) return 0;
    float c[48];
    for (int f = 0; f < 48; ++f) c[f] = rgb[48 * k + f];
    mask_empty(c, occ16);
    return encode16(c);
}

}  // namespace dxt1
}  // namespace vx
