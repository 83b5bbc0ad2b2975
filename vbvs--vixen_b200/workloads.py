"""Seeded synthetic workloads for the ESVO ray-casting path.

The reference measures on procedural scenes only (application/benchmark/
benchmark_config.json:49-80, RenderGraph/src/Data/SceneGenerator.cpp); the
scenes here have the shapes, sizes and fill fractions of the benchmark
configurations this library is measured on:

  cfg1  256^3 (octree depth 8), value noise (spacing 32, 4 octaves) at 10 %
        fill plus a one-voxel box shell; RGBA8 colour per voxel; 512x512
        pinhole camera, 60 deg, at the centre of the -Z face looking +Z.
        The face itself is shell, so the camera sits just inside it, at the
        centre of the face's middle voxel, (128.5, 128.5, 1.5).  (At exactly
        x = y = 128 every ray starts on an ESVO cell boundary and the
        reference traversal exits before reaching any voxel.)
  cfg2  1024^3 (depth 10), value noise (spacing 64, 5 octaves) at 50 % fill;
        DXT1 bricks with uniform random heads and index words; 1920x1080,
        70 deg, at a seeded empty voxel looking in a uniform random direction.
  cfg3  2048^3 (depth 11) urban lattice: 32x32 blocks, 8-voxel streets,
        heights uniform in [64, 1800]; DXT1 bricks; 3840x2160 primary rays
        plus one shadow ray per hit toward a seeded directional light.

Every input is produced on the host in binary32 so the oracle and the GPU see
the same bits.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import (VX_COLOR_DXT1, VX_COLOR_NONE, VX_COLOR_RGBA8, CameraPC, SceneArrays, build_dense, camera_rays,
               synth_dxt1, synth_noise, synth_rgba8, synth_urban)


def levels_for(R: int) -> int:
    """ceil(log2(R)) as VoxelSceneCacher::BuildOctree picks maxLevels (VoxelSceneCacher.cpp:525-528)."""
    return int(math.ceil(math.log2(R)))


def splitmix64(z: int) -> int:
    z = (z + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return z ^ (z >> 31)


def _f32(v):
    return np.asarray(v, np.float32)


def _normalize(v):
    v = _f32(v)
    d = np.float32((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2])
    return (v * (np.float32(1.0) / np.sqrt(d))).astype(np.float32)


def _cross(a, b):
    a, b = _f32(a), _f32(b)
    return _f32([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]])


def look_camera(pos, direction, fov_deg, width, height) -> CameraPC:
    d = _normalize(direction)
    up0 = _f32([0, 1, 0]) if abs(float(d[1])) < 0.99 else _f32([1, 0, 0])
    right = _normalize(_cross(d, up0))
    up = _cross(right, d)
    return CameraPC.make(pos, d, up, right, fov_deg, float(np.float32(width) / np.float32(height)))


@dataclass
class Workload:
    name: str
    R: int
    scene: SceneArrays
    bits: np.ndarray
    camera: CameraPC
    width: int
    height: int

    def rays(self, order: str = "rows") -> np.ndarray:
        """The camera's primary rays (vx_camera_rays).  order="rows": pixel y * width + x;
        order="tiled": the order vx_render gives them to warps (tile_order)."""
        r = camera_rays(self.camera, self.width, self.height)
        return r if order == "rows" else r[tile_order(self.width, self.height)]


def tile_order(width: int, height: int) -> np.ndarray:
    """Pixel indices in the order vx_render assigns them to threads: 32 x 8 tiles row by row,
    inside a tile eight 8 x 4 warp pieces (4 across, 2 down), inside a piece row-major;
    pixels outside the image are skipped."""
    tw, th = -(-width // 32), -(-height // 8)
    t = np.arange(tw * th * 256, dtype=np.int64)
    tile, thr = t // 256, t % 256
    warp, lane = thr // 32, thr % 32
    x = (tile % tw) * 32 + (warp % 4) * 8 + lane % 8
    y = (tile // tw) * 8 + (warp // 4) * 4 + lane // 8
    keep = (x < width) & (y < height)
    return (y * width + x)[keep].astype(np.int64)


def noise_scene(R, spacing, octaves, fill, seed, shell, color, max_levels=None):
    bits = synth_noise(R, spacing, octaves, fill, seed, shell)
    return scene_from_bits(bits, R, color, seed, max_levels), bits


def scene_from_bits(bits, R, color, seed, max_levels=None) -> SceneArrays:
    a = build_dense(bits, R, max_levels or levels_for(R))
    if color == "rgba8":
        a.color_kind, a.brick_color = VX_COLOR_RGBA8, synth_rgba8(a.brick_coord, seed ^ 0xC0105)
    elif color == "dxt1":
        a.color_kind, a.brick_color = VX_COLOR_DXT1, synth_dxt1(a.brick_coord, seed ^ 0xD7C1)
    else:
        a.color_kind, a.brick_color = VX_COLOR_NONE, None
    return a


def config1(R: int = 256, width: int = 512, height: int = 512, seed: int = 1) -> Workload:
    """cfg1; R, width and height shrink it for fast parity tests."""
    spacing = max(4, 32 * R // 256)
    scene, bits = noise_scene(R, spacing, 4 if spacing >= 32 else 3, 0.10, seed, True, "rgba8")
    cam = look_camera([R / 2 + 0.5, R / 2 + 0.5, 1.5], [0, 0, 1], 60.0, width, height)
    return Workload(f"cfg1_noise{R}_rgba8_{width}x{height}", R, scene, bits, cam, width, height)


def empty_voxel_camera(bits, R, seed, fov, width, height) -> CameraPC:
    wpr = R // 64
    k = 0
    while True:
        h = splitmix64(seed * 1000003 + k)
        x, y, z = h % R, (h >> 20) % R, (h >> 40) % R
        w = int(bits[(z * R + y) * wpr + (x >> 6)])
        if not (w >> (x & 63)) & 1:
            break
        k += 1
    h1, h2 = splitmix64(seed ^ 0xA5A5A5A5), splitmix64(seed ^ 0x5A5A5A5A)
    u, v = (h1 >> 11) / float(1 << 53), (h2 >> 11) / float(1 << 53)
    cz = 1.0 - 2.0 * u
    r = math.sqrt(max(0.0, 1.0 - cz * cz))
    phi = 2.0 * math.pi * v
    d = [r * math.cos(phi), r * math.sin(phi), cz]
    return look_camera([x + 0.5, y + 0.5, z + 0.5], d, fov, width, height)


def config2(R: int = 1024, width: int = 1920, height: int = 1080, seed: int = 2, bits=None) -> Workload:
    """cfg2; bits may be supplied (e.g. generated on the GPU with the same definition)."""
    spacing = max(4, 64 * R // 1024)
    if bits is None:
        bits = synth_noise(R, spacing, 5 if spacing >= 64 else 3, 0.50, seed, False)
    scene = scene_from_bits(bits, R, "dxt1", seed)
    cam = empty_voxel_camera(bits, R, seed, 70.0, width, height)
    return Workload(f"cfg2_cave{R}_dxt1_{width}x{height}", R, scene, bits, cam, width, height)


def config3(R: int = 2048, width: int = 3840, height: int = 2160, seed: int = 3) -> Workload:
    hmin, hmax = (64, 1800) if R == 2048 else (max(1, R // 32), max(2, R * 1800 // 2048))
    bits = synth_urban(R, hmin, hmax, seed)
    scene = scene_from_bits(bits, R, "dxt1", seed)
    cam = look_camera([R * 0.5, R * 0.9, -R * 0.25], [0.05, -0.45, 1.0], 60.0, width, height)
    return Workload(f"cfg3_urban{R}_dxt1_{width}x{height}", R, scene, bits, cam, width, height)


def random_rays(n: int, R: float, seed: int, lo=-0.25, hi=1.25) -> np.ndarray:
    """Origins uniform in [lo*R, hi*R]^3, directions uniform on the sphere,
    plus axis-aligned and near-axis directions (every 7th / 11th ray)."""
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo * R, hi * R, size=(n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    axis = rng.integers(0, 3, size=n)
    sign = rng.choice(np.array([-1.0, 1.0], np.float32), size=n)
    k = np.arange(n)
    aa = (k % 7) == 3
    d[aa] = 0.0
    d[aa, axis[aa]] = sign[aa]
    na = (k % 11) == 5
    d[na] = np.float32(1e-6) * d[na]
    d[na, axis[na]] = sign[na]
    return np.concatenate([o, d], axis=1).astype(np.float32)


@dataclass
class SceneSpec:
    R: int
    kind: str      # "noise" or "urban"
    fill: float    # noise fill fraction (urban: 0.9 nominal)
    color: str     # "dxt1" or "rgba8"
    width: int
    height: int
    seed: int


def config4_specs(n_scenes: int = 64, seed: int = 4, r_range=(6, 10), res_lo=(256, 256), res_hi=(1920, 1080)):
    """cfg4 scene draws: R = 2^round(U[6,10]), density in {10,50,90} % (noise for 10/50,
    urban for 90), DXT1 for every other scene, resolution log-uniform between 256x256 and
    1920x1080 (one uniform draw t: w = 256*(1920/256)^t, h = 256*(1080/256)^t)."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n_scenes):
        R = 2 ** int(round(rng.uniform(*r_range)))
        fill = float(rng.choice([0.1, 0.5, 0.9]))
        t = rng.uniform(0.0, 1.0)
        w = int(round(res_lo[0] * (res_hi[0] / res_lo[0]) ** t))
        h = int(round(res_lo[1] * (res_hi[1] / res_lo[1]) ** t))
        specs.append(SceneSpec(R, "urban" if fill > 0.8 else "noise", fill, "dxt1" if i % 2 else "rgba8", w, h,
                               seed * 1000 + i))
    return specs


def build_spec(spec: SceneSpec, bits=None) -> Workload:
    R = spec.R
    if bits is None:
        if spec.kind == "noise":
            spacing = max(4, 64 * R // 1024)
            bits = synth_noise(R, spacing, 5 if spacing >= 64 else 3, spec.fill, spec.seed, False)
        else:
            bits = synth_urban(R, max(1, R // 32), max(2, R * 1800 // 2048), spec.seed)
    scene = scene_from_bits(bits, R, spec.color, spec.seed)
    if spec.kind == "noise":
        cam = empty_voxel_camera(bits, R, spec.seed, 70.0, spec.width, spec.height)
    else:
        cam = look_camera([R * 0.5, R * 0.9, -R * 0.25], [0.05, -0.45, 1.0], 60.0, spec.width, spec.height)
    return Workload(f"cfg4_{spec.kind}{R}_{spec.color}_{spec.width}x{spec.height}", R, scene, bits, cam,
                    spec.width, spec.height)


def bounce_rays_reference(rays: np.ndarray, hits: np.ndarray, seed: int, table: np.ndarray) -> np.ndarray:
    """vx_spawn_bounce_rays restated in numpy binary32 (used by the tests)."""
    n = rays.shape[0]
    out = np.zeros((2 * n, 6), np.float32)
    out[0::2, :3] = rays[:, :3]
    out[1::2, :3] = rays[:, :3]
    hit = (hits["flags"] & 1).astype(bool)
    o, d = rays[:, :3], rays[:, 3:]
    dd = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
    inv = np.float32(1.0) / np.sqrt(dd)
    org = (o + (d * inv[:, None]) * hits["t"][:, None]).astype(np.float32)
    axis = (hits["flags"].astype(np.int64) >> 1) & 3
    sgn = np.where(hits["flags"] & 8, np.float32(-1.0), np.float32(1.0)).astype(np.float32)
    rows = np.arange(n)
    org[rows, axis] = org[rows, axis] + sgn * np.float32(0.001)
    for k in range(2):
        j = np.array([splitmix64(seed ^ splitmix64((i << 1) | k)) & 4095 for i in range(n)], np.int64)
        u, v, w = table[j, 0], table[j, 1], table[j, 2] * sgn
        dirs = np.stack([u, v, w], 1)
        dirs[axis == 0] = np.stack([w, u, v], 1)[axis == 0]
        dirs[axis == 1] = np.stack([v, w, u], 1)[axis == 1]
        sel = hit
        out[2 * rows[sel] + k, :3] = org[sel]
        out[2 * rows[sel] + k, 3:] = dirs[sel]
    return out


@dataclass
class DiffWorkload:
    wl: Workload
    kind: int
    attr: np.ndarray          # FP32 attributes (VX_DIFF_* layout)
    target_attr: np.ndarray   # attr + N(0, 0.05): the colours the target images are rendered from
    dxt_idx: np.ndarray | None
    views: list


def config5(R: int = 512, views: int = 16, width: int = 512, height: int = 512, kind: int = 0, seed: int = 5,
            bits=None) -> DiffWorkload:
    """cfg5: 512^3 value-noise scene at 30 % fill (spacing 32, 4 octaves); FP32 per-voxel RGB
    (kind 0) or FP32 DXT1 endpoints with fixed selectors (kind 1); `views` pinhole views on a
    seeded orbit around the grid centre, looking at it; targets rendered from the attributes
    plus N(0, 0.05)."""
    spacing = max(4, 32 * R // 512)
    if bits is None:
        bits = synth_noise(R, spacing, 4 if spacing >= 32 else 3, 0.30, seed, False)
    scene = scene_from_bits(bits, R, None, seed)
    rng = np.random.default_rng(seed)
    B = scene.brick_count
    if kind == 0:
        attr = rng.random(B * 512 * 3, dtype=np.float32)
        idx = None
    else:
        attr = rng.random(B * 32 * 6, dtype=np.float32)
        idx = rng.integers(0, 2 ** 32, size=B * 32, dtype=np.uint64).astype(np.uint32)
    target = (attr + rng.normal(0.0, 0.05, size=attr.shape).astype(np.float32)).astype(np.float32)
    c = np.float32(R / 2)
    cams = []
    phase = rng.uniform(0, 2 * np.pi)
    for v in range(views):
        th = phase + 2 * np.pi * v / views
        pos = [c + 0.95 * R * np.cos(th), c + R * rng.uniform(-0.3, 0.3), c + 0.95 * R * np.sin(th)]
        cams.append(look_camera(pos, [c - pos[0], c - pos[1], c - pos[2]], 60.0, width, height))
    wl = Workload(f"cfg5_noise{R}_{'rgb' if kind == 0 else 'dxt1ep'}_{views}x{width}x{height}", R, scene, bits,
                  cams[0], width, height)
    return DiffWorkload(wl, kind, attr, target, idx, cams)


def lambert_k64(flags: np.ndarray) -> np.ndarray:
    """Lambert factor of Lighting.glsl:19-28 per hit flag, in double."""
    L = np.array([1.0, 1.0, -1.0]) / np.sqrt(3.0)
    axis = (flags.astype(np.int64) >> 1) & 3
    sgn = np.where(flags & 8, -1.0, 1.0)
    return 0.3 + np.maximum(sgn * L[axis], 0.0) * 0.7


def dxt_weights64(idx: np.ndarray, block: np.ndarray, voxel: np.ndarray):
    sel = (idx[block].astype(np.int64) >> (2 * (voxel.astype(np.int64) & 15))) & 3
    w0 = np.array([1.0, 0.0, 2.0 / 3.0, 1.0 / 3.0])[sel]
    w1 = np.array([0.0, 1.0, 1.0 / 3.0, 2.0 / 3.0])[sel]
    return w0, w1


def adjoint_reference64(dw: DiffWorkload, records, targets) -> np.ndarray:
    """FP64 gradient of the L2 loss, replaying the forward records (brick, voxel, normal) with
    the colour math in double."""
    grad = np.zeros(dw.attr.shape[0], np.float64)
    attr = dw.attr.astype(np.float64)
    for rec, tgt in zip(records, targets):
        hit = (rec["flags"] & 1).astype(bool)
        br, vx_, fl = rec["brick"][hit].astype(np.int64), rec["voxel"][hit].astype(np.int64), rec["flags"][hit]
        k = lambert_k64(fl)
        t = tgt.reshape(-1, 3)[hit].astype(np.float64)
        if dw.kind == 0:
            base = (br * 512 + vx_) * 3
            for ch in range(3):
                pix = attr[base + ch] * k
                np.add.at(grad, base + ch, 2.0 * (pix - t[:, ch]) * k)
        else:
            blk = br * 32 + (vx_ >> 4)
            w0, w1 = dxt_weights64(dw.dxt_idx, blk, vx_)
            for ch in range(3):
                pix = (w0 * attr[blk * 6 + ch] + w1 * attr[blk * 6 + 3 + ch]) * k
                g = 2.0 * (pix - t[:, ch]) * k
                np.add.at(grad, blk * 6 + ch, w0 * g)
                np.add.at(grad, blk * 6 + 3 + ch, w1 * g)
    return grad


def light_dir(seed: int) -> np.ndarray:
    """Seeded directional light for cfg3 shadow rays: above the horizon (y > 0.3), normalised
    in binary32."""
    rng = np.random.default_rng(seed ^ 0x116)
    v = rng.normal(size=3)
    v[1] = abs(v[1]) + 0.3 * np.linalg.norm(v)
    return _normalize(v.astype(np.float32))
