"""Generates the committed golden vectors in this directory.

The reference ships no golden blocks or hit records (its tests assert
tolerances only) and cannot be built here, so these vectors come from the CPU
oracle (oracle/vx_oracle.cpp).  They pin the oracle against drift and give the
GPU tests a fixed expected output that does not need the oracle at run time.

Run from the repository root:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import kat_cases as K  # noqa: E402
import vx_oracle as vo  # noqa: E402

FIELDS = ["t", "brick", "node", "voxel", "flags", "iters", "grid_reads", "dda_steps", "key"]
LOD_PARAMS = [(0.0, 0.0), (0.0, 0.02), (0.0, 0.1), (0.5, 0.05)]


def rays_for(case_world_min, extent, n, seed):
    rng = np.random.default_rng(seed)
    o = rng.uniform(-0.5 * extent, 1.5 * extent, size=(n, 3)).astype(np.float32) + np.asarray(case_world_min,
                                                                                               np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    return np.concatenate([o, d], 1).astype(np.float32)


def main():
    out = {}
    # 1. KAT scenes: the KAT ray plus 256 random rays each.
    for i, c in enumerate(K.CASES):
        s = vo.OracleScene.from_positions(c.voxels, c.world_min, c.world_max, c.depth)
        extent = float(np.max(np.asarray(c.world_max) - np.asarray(c.world_min)))
        rays = np.concatenate([np.array([list(c.origin) + list(c.direction)], np.float32),
                               rays_for(c.world_min, extent, 256, 1000 + i)])
        h = s.cast_rays(rays, c.tmin, c.tmax)
        out[f"kat_{c.name}_rays"] = rays
        for f in FIELDS:
            out[f"kat_{c.name}_{f}"] = h[f]
    # 2. A 64^3 grid with random occupancy (bits stored) and 4096 rays.
    rng = np.random.default_rng(77)
    R = 64
    bits = (rng.integers(0, 2 ** 63, size=R * R * (R // 64), dtype=np.int64).view(np.uint64) &
            rng.integers(0, 2 ** 63, size=R * R * (R // 64), dtype=np.int64).view(np.uint64) &
            rng.integers(0, 2 ** 63, size=R * R * (R // 64), dtype=np.int64).view(np.uint64))
    s = vo.OracleScene.from_dense(bits, R, 6)
    rays = rays_for((0, 0, 0), R, 4096, 78)
    h = s.cast_rays(rays)
    out["dense64_bits"] = bits
    out["dense64_rays"] = rays
    for f in FIELDS:
        out[f"dense64_{f}"] = h[f]
    ex = s.export()
    for k, v in ex.items():
        out[f"dense64_{k}"] = v
    # 3b. castRayWithLOD on the same grid and rays at four cone sizes
    #     ({orig, dir}: off, castRayLOD-style spreads, and one with an origin size).
    out["dense64_lod_params"] = np.array(LOD_PARAMS, np.float32)
    for j, lod in enumerate(LOD_PARAMS):
        h = s.cast_rays_lod(rays, lod)
        for f in FIELDS + ["scale"]:
            out[f"dense64_lod{j}_{f}"] = h[f]
    # 3. DXT1 decode of 256 random blocks.
    blocks = rng.integers(0, 2 ** 63, size=256, dtype=np.int64).view(np.uint64) ^ np.uint64(0x8000000000000000)
    out["dxt_blocks"] = blocks
    out["dxt_texels"] = np.stack([vo.dxt1_decode_block(int(b)) for b in blocks])
    np.savez_compressed(os.path.join(HERE, "oracle_golden.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
