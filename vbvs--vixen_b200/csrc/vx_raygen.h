// vx_raygen.h - primary-ray generation shared by the host (vx_camera_rays)
// and the device (vx_render), so both produce identical bits.
//
// Restates getRayDir (shaders/RayGeneration.glsl:61-71) and the pixel uv of
// VoxelRayMarch.comp:453-455 in binary32, one operation at a time:
//   uv  = (pixel + 0.5) / size
//   ndc = uv * 2 - 1, ndc.y = -ndc.y
//   dir = (camDir + ((camRight * ndc.x) * tanHalf) * aspect) + (camUp * ndc.y) * tanHalf
//   dir = dir * (1 / sqrt((dir.x*dir.x + dir.y*dir.y) + dir.z*dir.z))
// tanHalf = tan(radians(fov/2)) is evaluated once on the host.
#pragma once

#include "vx_internal.h"

namespace vx {

__host__ __device__ inline void camera_ray(const CameraDev& c, uint32_t px, uint32_t py, uint32_t w, uint32_t h,
                                           vx_ray& r, float* uv_y_out) {
    float u = (float(px) + 0.5f) / float(w);
    float v = (float(py) + 0.5f) / float(h);
    float nx = u * 2.0f - 1.0f;
    float ny = v * 2.0f - 1.0f;
    ny = -ny;
    float d[3];
    for (int i = 0; i < 3; ++i) {
        float a = c.dir[i] + ((c.right[i] * nx) * c.tan_half_fov) * c.aspect;
        float b = (c.up[i] * ny) * c.tan_half_fov;
        d[i] = a + b;
    }
    float dd = (d[0] * d[0] + d[1] * d[1]) + d[2] * d[2];
    float inv = 1.0f / sqrtf(dd);
    r.ox = c.pos[0];
    r.oy = c.pos[1];
    r.oz = c.pos[2];
    r.dx = d[0] * inv;
    r.dy = d[1] * inv;
    r.dz = d[2] * inv;
    if (uv_y_out) *uv_y_out = v;
}

}  // namespace vx
