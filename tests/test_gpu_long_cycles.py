"""Rays caught in a state that repeats after more than two iterations (needs a B200).

The reference loop runs such rays to its 500-iteration cap.  The kernels compare the loop state
and the stack with a checkpoint taken at iterations 16, 32, 64, ..., and on a proven repeat
skip the whole cycles the cap leaves room for.  The records and the reference-loop counters
(iterations, grid reads, DDA steps) of every capped ray must still equal the oracle's, which
runs every iteration; checked through the plain kernel and the batched kernels (static lanes
with the stack in shared and in local memory, refilling lanes), on primary and bounce rays.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SEEDS = (4, 5, 6)
FIELDS = ("flags", "brick", "node", "voxel", "iters", "grid_reads", "dda_steps")


def _frame(vx, W, seed):
    import torch
    specs = W.config4_specs(8, seed=seed, r_range=(6, 8), res_lo=(192, 128), res_hi=(640, 480))
    wls = [W.build_spec(sp) for sp in specs]
    scenes = [vx.Scene(w.scene) for w in wls]
    rays = [w.rays(order="tiled") for w in wls]
    begin = np.concatenate([[0], np.cumsum([r.shape[0] for r in rays])]).astype(np.int64)
    d_rays = torch.from_numpy(np.concatenate(rays)).cuda()
    d_begin = torch.from_numpy(begin.astype(np.int32)).cuda()
    n = d_rays.shape[0]
    batch = vx.Batch(scenes)
    ph = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    batch.cast(d_rays, d_begin, ph)
    bounce = torch.zeros((2 * n, 6), dtype=torch.float32, device="cuda")
    vx.spawn_bounce_rays(d_rays, ph, 17, bounce)
    torch.cuda.synchronize()
    allr = torch.cat([d_rays, bounce])
    # scene ranges of the primary rays, then of the bounce rays
    ranges = [(int(begin[i]), int(begin[i + 1])) for i in range(len(wls))] + \
             [(n + 2 * int(begin[i]), n + 2 * int(begin[i + 1])) for i in range(len(wls))]
    allbegin = np.concatenate([begin, n + 2 * begin[1:]])
    return wls, scenes, allr, ranges, allbegin, batch


def _records(vx, hits, counters):
    g = hits.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1)
    c = counters.cpu().numpy().view(vx.COUNTER_DTYPE).reshape(-1)
    return g, c


def test_long_cycles_equal_oracle(vx, vo, cuda):
    import torch
    from vx_b200 import workloads as W
    skipped_total = capped_total = 0
    for seed in SEEDS:
        wls, scenes, allr, ranges, allbegin, _ = _frame(vx, W, seed)
        S = len(wls)
        # one batch over every (scene, ray set) range: primary ranges then bounce ranges
        batch = vx.Batch(scenes + scenes)
        d_begin = torch.from_numpy(allbegin.astype(np.int32)).cuda()
        m = allr.shape[0]
        results = {}
        for tun in ((256, 32, 1, 0, 0), (128, 64, 0, 0, 0), (256, 32, 1, 0, 24), (256, 128, 0, 16, 0)):
            hits = torch.zeros((m, 4), dtype=torch.int32, device="cuda")
            cnt = torch.zeros((m, 4), dtype=torch.int32, device="cuda")
            batch.set_tuning(*tun)
            batch.cast(allr, d_begin, hits, cnt)
            torch.cuda.synchronize()
            results[tun] = _records(vx, hits, cnt)
        plain_h = torch.zeros((m, 4), dtype=torch.int32, device="cuda")
        plain_c = torch.zeros((m, 4), dtype=torch.int32, device="cuda")
        for k, (a, b) in enumerate(ranges):
            scenes[k % S].cast_rays_dev(allr[a:b], plain_h[a:b], None, plain_c[a:b])
        torch.cuda.synchronize()
        results["plain"] = _records(vx, plain_h, plain_c)
        g0, c0 = results["plain"]
        for key, (g, c) in results.items():  # every kernel writes the same records and counters
            np.testing.assert_array_equal(g.view(np.uint32).reshape(-1), g0.view(np.uint32).reshape(-1), err_msg=str(key))
            for f in ("iters", "grid_reads", "dda_steps"):
                np.testing.assert_array_equal(c[f], c0[f], err_msg=f"{key} {f}")
        capped = c0["iters"] >= 500
        skipped = capped & (c0["run_iters"] > 16) & (c0["run_iters"] < 500)
        skipped_total += int(skipped.sum())
        capped_total += int(capped.sum())
        rays_np = allr.cpu().numpy()
        for k, (a, b) in enumerate(ranges):
            sel = np.flatnonzero(capped[a:b]) + a
            sel = np.concatenate([sel, np.arange(a, b, 97)])  # and a sample of the rest
            if sel.size == 0:
                continue
            w = wls[k % S]
            o = vo.OracleScene.from_dense(w.bits, w.R, w.scene.max_levels).cast_rays(rays_np[sel])
            got = {"flags": g0["flags"][sel].astype(np.uint32) & 0xFF, "brick": g0["brick"][sel],
                   "node": g0["node"][sel], "voxel": g0["voxel"][sel].astype(np.uint32),
                   "iters": c0["iters"][sel].astype(np.uint32), "grid_reads": c0["grid_reads"][sel].astype(np.uint32),
                   "dda_steps": c0["dda_steps"][sel].astype(np.uint32)}
            for f in FIELDS:
                want = o[f].astype(np.uint32)
                if f == "flags":
                    want = want & 0xFF
                bad = np.flatnonzero(got[f] != want)
                assert bad.size == 0, f"seed {seed} range {k} {f}: {bad.size} of {sel.size} differ, first ray " \
                                      f"{sel[bad[0]]}: gpu {got[f][bad[0]]} oracle {want[bad[0]]}"
            hit = (o["flags"] & 1).astype(bool)
            np.testing.assert_array_equal(g0["t"][sel][hit].view(np.uint32), o["t"][hit].view(np.uint32))
    assert capped_total > 0
    assert skipped_total > 0, "no ray took the long-cycle skip: the test scenes no longer exercise it"
