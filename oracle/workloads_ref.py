"""The benchmark frames rebuilt on the oracle side, without the product library.

TEST INFRASTRUCTURE ONLY: used by the CPU baseline and the reference arm of
bench.py and by the tests.  It restates the seeded workload definitions of the
product's workloads module (scene draws, cameras, ray order) and produces the
scenes' occupancy bits, the primary rays and the secondary rays with the
oracle's own functions (vx_oracle_synth.cpp, vxo_camera_rays), so a run that
uses it never loads libvx.so.  tests/test_oracle_workloads.py checks every
piece against the product's bits.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

import vx_oracle as vo

M64 = 0xFFFFFFFFFFFFFFFF


def splitmix64(z: int) -> int:
    z = (z + 0x9E3779B97F4A7C15) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def levels_for(R: int) -> int:
    """maxLevels = ceil(log2 R), as VoxelSceneCacher::BuildOctree picks it (VoxelSceneCacher.cpp:525-528)."""
    return int(math.ceil(math.log2(R)))


def _unit(v):
    v = np.asarray(v, np.float32)
    d = np.float32((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2])
    return (v * (np.float32(1.0) / np.sqrt(d))).astype(np.float32)


def _cross(a, b):
    a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
    return np.asarray([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]],
                      np.float32)


def look_camera(pos, direction, fov_deg, width, height) -> np.ndarray:
    """Push constants (16 words, VoxelRayMarch.comp:85-94) of a camera at pos looking along
    direction, with right = normalize(d x up0) and up = right x d (up0 = +y unless d is near it)."""
    d = _unit(direction)
    up0 = np.asarray([0, 1, 0], np.float32) if abs(float(d[1])) < 0.99 else np.asarray([1, 0, 0], np.float32)
    right = _unit(_cross(d, up0))
    up = _cross(right, d)
    pc = np.zeros(16, np.float32)
    pc[0:3] = np.asarray(pos, np.float32)
    pc[4:7] = d
    pc[7] = np.float32(fov_deg)
    pc[8:11] = up
    pc[11] = np.float32(width) / np.float32(height)
    pc[12:15] = right
    return pc


def empty_voxel_camera(bits, R, seed, fov, width, height) -> np.ndarray:
    """A camera at the centre of the first empty voxel of a seeded sequence, looking in a seeded
    uniform direction."""
    wpr = R // 64
    k = 0
    while True:
        h = splitmix64(seed * 1000003 + k)
        x, y, z = h % R, (h >> 20) % R, (h >> 40) % R
        if not (int(bits[(z * R + y) * wpr + (x >> 6)]) >> (x & 63)) & 1:
            break
        k += 1
    u = (splitmix64(seed ^ 0xA5A5A5A5) >> 11) / float(1 << 53)
    v = (splitmix64(seed ^ 0x5A5A5A5A) >> 11) / float(1 << 53)
    cz = 1.0 - 2.0 * u
    r = math.sqrt(max(0.0, 1.0 - cz * cz))
    phi = 2.0 * math.pi * v
    return look_camera([x + 0.5, y + 0.5, z + 0.5], [r * math.cos(phi), r * math.sin(phi), cz], fov, width, height)


def tile_order(width: int, height: int) -> np.ndarray:
    """Pixel order of the render kernel: 32 x 8 tiles row by row, eight 8 x 4 warp pieces per tile
    (4 across, 2 down), row-major inside a piece; pixels outside the image skipped."""
    tw, th = -(-width // 32), -(-height // 8)
    t = np.arange(tw * th * 256, dtype=np.int64)
    tile, thr = t // 256, t % 256
    warp, lane = thr // 32, thr % 32
    x = (tile % tw) * 32 + (warp % 4) * 8 + lane % 8
    y = (tile // tw) * 8 + (warp // 4) * 4 + lane // 8
    keep = (x < width) & (y < height)
    return (y * width + x)[keep].astype(np.int64)


def noise_bits(R, spacing, octaves, fill, seed, shell=False, threads=0) -> np.ndarray:
    out = np.zeros(R * R * (R // 64), np.uint64)
    if vo.lib().vxo_synth_noise(R, spacing, octaves, float(fill), seed, int(shell), vo._ptr(out), threads) != 0:
        raise ValueError("vxo_synth_noise: bad arguments")
    return out


def urban_bits(R, hmin, hmax, seed) -> np.ndarray:
    out = np.zeros(R * R * (R // 64), np.uint64)
    if vo.lib().vxo_synth_urban(R, hmin, hmax, seed, vo._ptr(out)) != 0:
        raise ValueError("vxo_synth_urban: bad arguments")
    return out


def bounce_table() -> np.ndarray:
    out = np.zeros(4096 * 3, np.float32)
    vo.lib().vxo_bounce_table(vo._ptr(out))
    return out.reshape(4096, 3)


def spawn_bounce(rays, hits, seed, index=None) -> np.ndarray:
    """Two bounce rays per ray from the oracle's hit records (2n x 6); index: each ray's
    position in its frame (default 0..n-1)."""
    rays = np.ascontiguousarray(rays, np.float32)
    hits = np.ascontiguousarray(hits)
    idx = None if index is None else np.ascontiguousarray(index, np.uint64)
    out = np.zeros((2 * rays.shape[0], 6), np.float32)
    vo.lib().vxo_spawn_rays(vo._ptr(rays), vo._ptr(hits), vo._ptr(idx), rays.shape[0], 0, seed, None, vo._ptr(out))
    return out


def spawn_shadow(rays, hits, light) -> np.ndarray:
    rays = np.ascontiguousarray(rays, np.float32)
    hits = np.ascontiguousarray(hits)
    L = np.ascontiguousarray(light, np.float32)
    out = np.zeros((rays.shape[0], 6), np.float32)
    vo.lib().vxo_spawn_rays(vo._ptr(rays), vo._ptr(hits), None, rays.shape[0], 1, 0, vo._ptr(L), vo._ptr(out))
    return out


@dataclass
class Frame:
    """One camera over one scene: occupancy bits, the camera and its primary rays (tiled order)."""
    name: str
    R: int
    max_levels: int
    bits: np.ndarray
    pc: np.ndarray
    width: int
    height: int

    def rays(self, order: str = "tiled") -> np.ndarray:
        r = vo.camera_rays(self.pc, self.width, self.height)
        return r if order == "rows" else r[tile_order(self.width, self.height)]

    def scene(self):
        return vo.OracleScene.from_dense(self.bits, self.R, self.max_levels)


def cfg2(R=1024, width=1920, height=1080, seed=2, threads=0) -> Frame:
    """Cave: value noise (spacing 64 R / 1024, 5 octaves from spacing 64 up, else 3) at 50 % fill."""
    spacing = max(4, 64 * R // 1024)
    bits = noise_bits(R, spacing, 5 if spacing >= 64 else 3, 0.5, seed, False, threads)
    return Frame(f"cfg2_cave{R}", R, levels_for(R), bits, empty_voxel_camera(bits, R, seed, 70.0, width, height),
                 width, height)


def cfg3(R=2048, width=3840, height=2160, seed=3) -> Frame:
    hmin, hmax = (64, 1800) if R == 2048 else (max(1, R // 32), max(2, R * 1800 // 2048))
    bits = urban_bits(R, hmin, hmax, seed)
    pc = look_camera([R * 0.5, R * 0.9, -R * 0.25], [0.05, -0.45, 1.0], 60.0, width, height)
    return Frame(f"cfg3_urban{R}", R, levels_for(R), bits, pc, width, height)


def light_dir(seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed ^ 0x116)
    v = rng.normal(size=3)
    v[1] = abs(v[1]) + 0.3 * np.linalg.norm(v)
    return _unit(v.astype(np.float32))


@dataclass
class Spec:
    R: int
    kind: str
    fill: float
    color: str
    width: int
    height: int
    seed: int


def cfg4_specs(n_scenes=64, seed=4, r_range=(6, 10), res_lo=(256, 256), res_hi=(1920, 1080)):
    """The scene draws of the batched frame: R = 2^round(U[6,10]), fill in {10, 50, 90} %
    (noise for 10/50, urban for 90), DXT1 every other scene, resolution log-uniform."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_scenes):
        R = 2 ** int(round(rng.uniform(*r_range)))
        fill = float(rng.choice([0.1, 0.5, 0.9]))
        t = rng.uniform(0.0, 1.0)
        w = int(round(res_lo[0] * (res_hi[0] / res_lo[0]) ** t))
        h = int(round(res_lo[1] * (res_hi[1] / res_lo[1]) ** t))
        out.append(Spec(R, "urban" if fill > 0.8 else "noise", fill, "dxt1" if i % 2 else "rgba8", w, h,
                        seed * 1000 + i))
    return out


def cfg4_frame(spec: Spec, threads=0) -> Frame:
    R = spec.R
    if spec.kind == "noise":
        spacing = max(4, 64 * R // 1024)
        bits = noise_bits(R, spacing, 5 if spacing >= 64 else 3, spec.fill, spec.seed, False, threads)
        pc = empty_voxel_camera(bits, R, spec.seed, 70.0, spec.width, spec.height)
    else:
        bits = urban_bits(R, max(1, R // 32), max(2, R * 1800 // 2048), spec.seed)
        pc = look_camera([R * 0.5, R * 0.9, -R * 0.25], [0.05, -0.45, 1.0], 60.0, spec.width, spec.height)
    return Frame(f"cfg4_{spec.kind}{R}", R, levels_for(R), bits, pc, spec.width, spec.height)
