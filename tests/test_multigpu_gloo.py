"""Multi-GPU host logic on CPU with world_size 2 (gloo): the ray split covers
every ray exactly once, per-rank casts concatenate to the single-process
result, and the timing reduction is the max over ranks."""
import os
import socket

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_ray_range_partition():
    import importlib.util
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import load_vx
    load_vx()
    from vx_b200 import multigpu as M
    for n in (0, 1, 7, 1000, 2073600):
        for world in (1, 2, 3, 8):
            ranges = [M.ray_range(n, r, world) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
            sizes = [e - b for b, e in ranges]
            assert max(sizes) - min(sizes) <= 1
    assert M.rank_seed(2, 0) == 2 and M.rank_seed(2, 1) != M.rank_seed(2, 0)
    with pytest.raises(ValueError):
        M.ray_range(10, 2, 2)


def _worker(rank, world, port, out_dir):
    import sys
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import torch.distributed as dist
    from conftest import load_vx
    import vx_oracle as vo
    load_vx()
    from vx_b200 import multigpu as M
    from vx_b200 import workloads as W
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    wl = W.config1(R=64, width=48, height=40, seed=5)
    rays = wl.rays()
    b, e = M.ray_range(rays.shape[0], rank, world)
    hits = vo.OracleScene.from_dense(wl.bits, 64, wl.scene.max_levels).cast_rays(rays[b:e], threads=1)
    parts = [None] * world
    dist.all_gather_object(parts, hits.tobytes())
    tmax = M.max_over_ranks([1.0 + rank, 5.0 - rank])
    if rank == 0:
        np.save(os.path.join(out_dir, "gathered.npy"), np.frombuffer(b"".join(parts), dtype=hits.dtype))
        np.save(os.path.join(out_dir, "tmax.npy"), np.array(tmax))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_split_matches_single_process(vo, tmp_path):
    import multiprocessing as mp
    from vx_b200 import workloads as W
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    gathered = np.load(tmp_path / "gathered.npy")
    wl = W.config1(R=64, width=48, height=40, seed=5)
    whole = vo.OracleScene.from_dense(wl.bits, 64, wl.scene.max_levels).cast_rays(wl.rays(), threads=1)
    assert np.array_equal(gathered.view(np.uint8), whole.view(np.uint8))
    assert list(np.load(tmp_path / "tmax.npy")) == [2.0, 5.0]


def _adjoint_worker(rank, world, port, out_dir):
    import sys
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import torch
    import torch.distributed as dist
    from conftest import load_vx
    import vx_oracle as vo
    load_vx()
    from vx_b200 import multigpu as M
    from vx_b200 import workloads as W
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    dw = W.config5(R=64, views=5, width=32, height=24, kind=1, seed=8)
    o = vo.OracleScene.from_dense(dw.wl.bits, 64, dw.wl.scene.max_levels)
    b, e = M.view_range(len(dw.views), rank, world)
    rng = np.random.default_rng(100)
    targets = [rng.random((32 * 24, 3)).astype(np.float32) for _ in dw.views]
    recs = [o.cast_rays(W.camera_rays(pc, 32, 24), threads=1) for pc in dw.views[b:e]]
    g = torch.from_numpy(W.adjoint_reference64(dw, recs, targets[b:e]))
    dense = g.clone()
    M.allreduce_sum_(dense)
    np.save(os.path.join(out_dir, f"grad{rank}.npy"), dense.numpy())
    # the sparse exchange: only the entries this rank's records touch
    as_vx = [np.stack([r["t"].view(np.int32), r["brick"].view(np.int32), r["node"].view(np.int32),
                       (r["voxel"].astype(np.int64) | (r["flags"].astype(np.int64) << 16)).astype(np.int32)], 1)
             for r in recs]
    entries = M.touched_entries(torch.from_numpy(np.concatenate(as_vx)), kind=1)
    assert torch.all(g[torch.from_numpy(np.setdiff1d(np.arange(g.numel()), entries.numpy()))] == 0)
    M.sparse_allreduce_(g, entries)
    np.save(os.path.join(out_dir, f"sparse{rank}.npy"), g.numpy())
    np.save(os.path.join(out_dir, f"touched{rank}.npy"), np.array([entries.numel(), g.numel()]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_adjoint_split_views_allreduce(vo, tmp_path):
    """Views split over two gloo ranks, per-rank gradients summed by all-reduce: every rank
    holds the single-process gradient of all views."""
    import multiprocessing as mp
    from vx_b200 import workloads as W
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_adjoint_worker, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    dw = W.config5(R=64, views=5, width=32, height=24, kind=1, seed=8)
    o = vo.OracleScene.from_dense(dw.wl.bits, 64, dw.wl.scene.max_levels)
    rng = np.random.default_rng(100)
    targets = [rng.random((32 * 24, 3)).astype(np.float32) for _ in dw.views]
    recs = [o.cast_rays(W.camera_rays(pc, 32, 24), threads=1) for pc in dw.views]
    whole = W.adjoint_reference64(dw, recs, targets)
    assert np.count_nonzero(whole) > 0
    for r in range(2):
        np.testing.assert_allclose(np.load(tmp_path / f"grad{r}.npy"), whole, rtol=1e-12, atol=1e-12)
        # the sparse exchange gives the same sums, bit-identical on both ranks
        np.testing.assert_allclose(np.load(tmp_path / f"sparse{r}.npy"), whole, rtol=1e-12, atol=1e-12)
        touched, total = np.load(tmp_path / f"touched{r}.npy")
        assert 0 < touched < total / 4
    np.testing.assert_array_equal(np.load(tmp_path / "sparse0.npy"), np.load(tmp_path / "sparse1.npy"))
