// vx_palette.h - material-ID colours, shared by the host and the device.
//
// The reference's scenes store a material word per voxel (brickData,
// CashSystem/src/VoxelSceneCacher.cpp:500, 586-587) and turn it into a colour
// in two places, with two tables that disagree on ids 33-39:
//  - the uncompressed compute shader colours a hit with
//    getMaterialColor(voxelData & 0xFF) (shaders/Materials.glsl:18-60,
//    VoxelRayMarch.comp:188-192): ids 33-39 blend two stone tones by
//    mix(a, b, (id - 33) / 6);
//  - the compressed payload is encoded from MaterialIdToColor(id)
//    (SVO/src/SVORebuild.cpp:68-120, used at :679-700): ids 33-39 come from
//    a table.
// Both fall back to an HSV colour wheel for ids they do not list.  Paths are
// relative to the reference project's VIXEN/ directory.  Arithmetic is IEEE
// binary32 in source order (no contraction), so host and device agree bit
// for bit.
#pragma once

#include <stdint.h>

#include "vx_hd.h"

namespace vx {

struct Rgb {
    float r, g, b;
};

// The colour-wheel fallback of both tables for an id they do not list.
VX_HD Rgb palette_wheel(uint32_t id) {
    const float hue = float(id % 256u) / 256.0f;
    const float h = hue * 6.0f;
    const int i = int(h);
    const float f = h - float(i);
    const float p = 0.8f * 0.3f;
    const float q = 0.8f * (1.0f - 0.7f * f);
    const float t = 0.8f * (1.0f - 0.7f * (1.0f - f));
    switch (i) {
        case 0: return {0.8f, t, p};
        case 1: return {q, 0.8f, p};
        case 2: return {p, 0.8f, t};
        case 3: return {p, q, 0.8f};
        case 4: return {t, p, 0.8f};
        default: return {0.8f, p, q};
    }
}

// Ids both tables list with the same colour; false for the rest.
VX_HD bool palette_common(uint32_t id, Rgb& c) {
    switch (id) {
        case 1: c = {1.0f, 0.0f, 0.0f}; return true;     // Cornell box 1-20
        case 2: c = {0.0f, 1.0f, 0.0f}; return true;
        case 3: c = {0.9f, 0.9f, 0.9f}; return true;
        case 4: c = {0.85f, 0.85f, 0.85f}; return true;
        case 5: c = {0.95f, 0.95f, 0.95f}; return true;
        case 6: c = {0.8f, 0.8f, 0.8f}; return true;
        case 7: c = {0.4f, 0.4f, 0.4f}; return true;
        case 10: c = {0.8f, 0.6f, 0.2f}; return true;
        case 11: c = {0.6f, 0.8f, 0.9f}; return true;
        case 20: c = {1.0f, 0.98f, 0.9f}; return true;
        case 30: c = {0.5f, 0.45f, 0.4f}; return true;   // noise / tunnel 30-40
        case 31: c = {0.6f, 0.55f, 0.5f}; return true;
        case 32: c = {0.55f, 0.5f, 0.45f}; return true;
        case 40: c = {0.8f, 0.6f, 0.2f}; return true;
        case 50: c = {0.2f, 0.2f, 0.22f}; return true;   // cityscape 50-61
        case 60: c = {0.6f, 0.58f, 0.55f}; return true;
        case 61: c = {0.7f, 0.85f, 0.95f}; return true;
        default: return false;
    }
}

// getMaterialColor (shaders/Materials.glsl:18-60) of id = word & 0xFF;
// GLSL's mix(x, y, a) = x * (1 - a) + y * a.
VX_HD Rgb material_color_shader(uint32_t id) {
    Rgb c;
    if (palette_common(id, c)) return c;
    if (id >= 33u && id <= 39u) {
        const float t = float(id - 33u) / 6.0f;
        const float u = 1.0f - t;
        return {0.52f * u + 0.68f * t, 0.48f * u + 0.6f * t, 0.42f * u + 0.52f * t};
    }
    return palette_wheel(id);
}

// MaterialIdToColor (SVO/src/SVORebuild.cpp:68-120): the colour the
// compressed payload is encoded from.
VX_HD Rgb material_color_payload(uint32_t id) {
    Rgb c;
    if (palette_common(id, c)) return c;
    switch (id) {
        case 33: return {0.52f, 0.48f, 0.42f};
        case 34: return {0.48f, 0.44f, 0.38f};
        case 35: return {0.45f, 0.42f, 0.36f};
        case 36: return {0.58f, 0.52f, 0.46f};
        case 37: return {0.62f, 0.56f, 0.48f};
        case 38: return {0.65f, 0.58f, 0.5f};
        case 39: return {0.68f, 0.6f, 0.52f};
        default: return palette_wheel(id);
    }
}

}  // namespace vx
