"""Committed golden vectors (tests/golden/make_golden.py).

CPU: the oracle reproduces every vector bit for bit.  GPU: the kernel
reproduces the 64^3 dense-grid vectors from the committed device buffers alone.
"""
import os

import numpy as np
import pytest

import kat_cases as K

HERE = os.path.dirname(os.path.abspath(__file__))
FIELDS = ["t", "brick", "node", "voxel", "flags", "iters", "grid_reads", "dda_steps", "key"]


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(HERE, "golden", "oracle_golden.npz"))


def _eq(a, b, label):
    a, b = np.asarray(a), np.asarray(b)
    if a.dtype.kind == "f":
        a, b = a.view(np.uint32), b.view(np.uint32)
    np.testing.assert_array_equal(a, b, err_msg=label)


@pytest.mark.parametrize("case", K.CASES, ids=[c.name for c in K.CASES])
def test_oracle_reproduces_kat_golden(vo, golden, case):
    s = vo.OracleScene.from_positions(case.voxels, case.world_min, case.world_max, case.depth)
    h = s.cast_rays(golden[f"kat_{case.name}_rays"], case.tmin, case.tmax)
    for f in FIELDS:
        _eq(h[f], golden[f"kat_{case.name}_{f}"], f"{case.name}.{f}")


def test_oracle_reproduces_dense_golden(vo, golden):
    s = vo.OracleScene.from_dense(golden["dense64_bits"], 64, 6)
    h = s.cast_rays(golden["dense64_rays"])
    for f in FIELDS:
        _eq(h[f], golden[f"dense64_{f}"], f)
    for k, v in s.export().items():
        _eq(v, golden[f"dense64_{k}"], k)


def test_oracle_reproduces_dxt_golden(vo, golden):
    for b, want in zip(golden["dxt_blocks"], golden["dxt_texels"]):
        _eq(vo.dxt1_decode_block(int(b)), want, hex(int(b)))


def test_builder_reproduces_dense_golden(vx, golden):
    a = vx.build_dense(golden["dense64_bits"], 64, 6)
    for k in ["nodes", "node_brick", "grid_lookup", "brick_coord", "brick_occ"]:
        _eq(getattr(a, k), golden[f"dense64_{k}"], k)


@pytest.mark.gpu
def test_kernel_reproduces_dense_golden(vx, golden, cuda):
    import torch
    a = vx.SceneArrays((0.0, 0.0, 0.0), (64.0, 64.0, 64.0), 6, 8, golden["dense64_nodes"],
                       golden["dense64_node_brick"], golden["dense64_grid_lookup"], golden["dense64_brick_coord"],
                       golden["dense64_brick_occ"])
    s = vx.Scene(a)
    rays = golden["dense64_rays"]
    n = rays.shape[0]
    r = torch.from_numpy(np.ascontiguousarray(rays)).cuda()
    hits = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    cnt = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    s.cast_rays_dev(r, hits, None, cnt)
    torch.cuda.synchronize()
    g = hits.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1)
    c = cnt.cpu().numpy().view(vx.COUNTER_DTYPE).reshape(-1)
    hit = (golden["dense64_flags"] & 1).astype(bool)
    _eq(g["flags"].astype(np.uint32), golden["dense64_flags"], "flags")
    _eq(g["t"][hit], golden["dense64_t"][hit], "t")
    _eq(g["brick"], golden["dense64_brick"], "brick")
    _eq(g["node"], golden["dense64_node"], "node")
    _eq(g["voxel"].astype(np.uint32), golden["dense64_voxel"], "voxel")
    _eq(c["iters"].astype(np.uint32), golden["dense64_iters"], "iters")
    _eq(c["dda_steps"].astype(np.uint32), golden["dense64_dda_steps"], "dda_steps")


def test_oracle_reproduces_lod_golden(vo, golden):
    s = vo.OracleScene.from_dense(golden["dense64_bits"], 64, 6)
    for j, lod in enumerate(golden["dense64_lod_params"]):
        h = s.cast_rays_lod(golden["dense64_rays"], tuple(float(v) for v in lod))
        for f in FIELDS + ["scale"]:
            _eq(h[f], golden[f"dense64_lod{j}_{f}"], f"lod{j}.{f}")


@pytest.mark.gpu
@pytest.mark.parametrize("j", range(4))
def test_kernel_reproduces_lod_golden(vx, golden, cuda, j):
    """castRayWithLOD on the committed device buffers: every field, including
    the LOD hits' distance bits, cell scale and parent descriptor."""
    import torch
    a = vx.SceneArrays((0.0, 0.0, 0.0), (64.0, 64.0, 64.0), 6, 8, golden["dense64_nodes"],
                       golden["dense64_node_brick"], golden["dense64_grid_lookup"], golden["dense64_brick_coord"],
                       golden["dense64_brick_occ"])
    s = vx.Scene(a)
    rays = golden["dense64_rays"]
    n = rays.shape[0]
    r = torch.from_numpy(np.ascontiguousarray(rays)).cuda()
    hits = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    cnt = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    lod = tuple(float(v) for v in golden["dense64_lod_params"][j])
    s.cast_rays_dev(r, hits, None, cnt, lod=lod)
    torch.cuda.synchronize()
    g = hits.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1)
    c = cnt.cpu().numpy().view(vx.COUNTER_DTYPE).reshape(-1)
    p = f"dense64_lod{j}_"
    hit = (golden[p + "flags"] & 1).astype(bool)
    assert hit.any()
    _eq(g["flags"].astype(np.uint32), golden[p + "flags"], "flags")
    _eq(g["t"][hit], golden[p + "t"][hit], "t")
    _eq(g["brick"], golden[p + "brick"], "brick")
    _eq(g["node"], golden[p + "node"], "node")
    _eq(g["voxel"].astype(np.uint32), golden[p + "voxel"], "voxel")
    _eq(g["scale"].astype(np.int32), golden[p + "scale"], "scale")
    _eq(c["iters"].astype(np.uint32), golden[p + "iters"], "iters")
    _eq(c["grid_reads"].astype(np.uint32), golden[p + "grid_reads"], "grid_reads")
    _eq(c["dda_steps"].astype(np.uint32), golden[p + "dda_steps"], "dda_steps")
