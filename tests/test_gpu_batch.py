"""Batched persistent kernel, secondary-ray spawn and the frame CUDA graph
(needs a B200).  The batched cast must return exactly the plain kernel's hits
for every scene, and the plain kernel's are checked against the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _small_specs(W, n=10, seed=11):
    return W.config4_specs(n, seed=seed, r_range=(6, 7.4), res_lo=(48, 40), res_hi=(160, 96))


def _setup(vx, W, n=10, seed=11):
    import torch
    wls = [W.build_spec(s) for s in _small_specs(W, n, seed)]
    scenes = [vx.Scene(w.scene) for w in wls]
    rays = [w.rays() for w in wls]
    begin = np.concatenate([[0], np.cumsum([r.shape[0] for r in rays])]).astype(np.uint32)
    allr = np.concatenate(rays).astype(np.float32)
    return wls, scenes, rays, begin, allr, torch.from_numpy(allr).cuda(), torch.from_numpy(begin.astype(np.int32)).cuda()


def _direction_bin(rows):
    """The compaction's direction bin of rays {o, d}: octant * 6 + the order of the axes by |d|
    (major axis, then whether the minor one follows it cyclically)."""
    d = rows[:, 3:6]
    ax, ay, az = np.abs(d).T
    octant = (d[:, 0] > 0).astype(np.int64) | ((d[:, 1] > 0).astype(np.int64) << 1) | \
        ((d[:, 2] > 0).astype(np.int64) << 2)
    major = np.where((ax >= ay) & (ax >= az), 0, np.where(ay >= az, 1, 2))
    minor = np.where((ax < ay) & (ax < az), 0, np.where(ay < az, 1, 2))
    assert np.all(major != minor)
    return octant * 6 + major * 2 + (minor != (major + 1) % 3).astype(np.int64)


def _plain(vx, scenes, rays, begin, d_rays):
    import torch
    n = d_rays.shape[0]
    hits = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    for i, s in enumerate(scenes):
        a, b = int(begin[i]), int(begin[i + 1])
        s.cast_rays_dev(d_rays[a:b], hits[a:b])
    torch.cuda.synchronize()
    return hits


@pytest.mark.parametrize("block,k,smem,refill,budget", [
    (256, 128, 1, 0, 0), (128, 32, 1, 0, 0), (256, 64, 0, 0, 0), (128, 512, 0, 0, 0),
    (256, 32, 1, 16, 0), (128, 64, 1, 8, 0), (256, 128, 0, 24, 0), (256, 32, 1, 32, 0), (128, 32, 0, 1, 0),
    # iteration budgets: every ray still running after 1, 3 or 8 iterations is cast again
    (256, 32, 1, 0, 1), (128, 64, 0, 0, 3), (256, 32, 1, 0, 8)])
def test_batch_equals_plain_and_oracle(vx, vo, cuda, block, k, smem, refill, budget):
    import torch
    from vx_b200 import workloads as W
    wls, scenes, rays, begin, allr, d_rays, d_begin = _setup(vx, W)
    plain = _plain(vx, scenes, rays, begin, d_rays)
    batch = vx.Batch(scenes)
    batch.set_tuning(block, k, smem, refill, budget)
    hits = torch.full_like(plain, -1)
    cnt = torch.zeros((allr.shape[0], 4), dtype=torch.int32, device="cuda")
    batch.cast(d_rays, d_begin, hits, cnt)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(hits.cpu().numpy(), plain.cpu().numpy())
    g = hits.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1)
    c = cnt.cpu().numpy().view(vx.COUNTER_DTYPE).reshape(-1)
    for i, w in enumerate(wls[:4]):
        a, b = int(begin[i]), int(begin[i + 1])
        oh = vo.OracleScene.from_dense(w.bits, w.R, w.scene.max_levels).cast_rays(rays[i])
        assert np.array_equal(g["brick"][a:b], oh["brick"]) and np.array_equal(g["node"][a:b], oh["node"])
        assert np.array_equal(g["flags"][a:b].astype(np.uint32), oh["flags"])
        assert np.array_equal(c["iters"][a:b].astype(np.uint32), oh["iters"])


def test_bounce_spawn_matches_reference_and_casts_exactly(vx, vo, cuda):
    import torch
    from vx_b200 import workloads as W
    wls, scenes, rays, begin, allr, d_rays, d_begin = _setup(vx, W, n=6, seed=12)
    hits = _plain(vx, scenes, rays, begin, d_rays)
    n = allr.shape[0]
    bounce = torch.zeros((2 * n, 6), dtype=torch.float32, device="cuda")
    vx.spawn_bounce_rays(d_rays, hits, 99, bounce)
    torch.cuda.synchronize()
    h = hits.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1)
    want = W.bounce_rays_reference(allr, h, 99, vx.bounce_table())
    np.testing.assert_array_equal(bounce.cpu().numpy().view(np.uint32), want.view(np.uint32))
    # bounce rays through the batched kernel vs the oracle, per scene
    bbegin = (2 * begin).astype(np.uint32)
    batch = vx.Batch(scenes)
    bh = torch.zeros((2 * n, 4), dtype=torch.int32, device="cuda")
    batch.cast(bounce, torch.from_numpy(bbegin.astype(np.int32)).cuda(), bh)
    torch.cuda.synchronize()
    g = bh.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1)
    for i, w in enumerate(wls):
        a, b = int(bbegin[i]), int(bbegin[i + 1])
        oh = vo.OracleScene.from_dense(w.bits, w.R, w.scene.max_levels).cast_rays(want[a:b])
        hit = (oh["flags"] & 1).astype(bool)
        assert np.array_equal(g["flags"][a:b].astype(np.uint32), oh["flags"])
        assert np.array_equal(g["brick"][a:b], oh["brick"]) and np.array_equal(g["voxel"][a:b].astype(np.uint32),
                                                                               oh["voxel"])
        assert np.array_equal(g["t"][a:b][hit].view(np.uint32), oh["t"][hit].view(np.uint32))


def test_shadow_spawn_matches_reference(vx, cuda):
    import torch
    from vx_b200 import workloads as W
    wls, scenes, rays, begin, allr, d_rays, d_begin = _setup(vx, W, n=3, seed=13)
    hits = _plain(vx, scenes, rays, begin, d_rays)
    n = allr.shape[0]
    L = np.array([0.3, 0.8, -0.52], np.float32)
    out = torch.zeros((n, 6), dtype=torch.float32, device="cuda")
    vx.spawn_shadow_rays(d_rays, hits, L, out)
    torch.cuda.synchronize()
    h = hits.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1)
    b = W.bounce_rays_reference(allr, h, 0, vx.bounce_table())[0::2]  # same origins
    hit = (h["flags"] & 1).astype(bool)
    got = out.cpu().numpy()
    np.testing.assert_array_equal(got[hit, :3].view(np.uint32), b[hit, :3].view(np.uint32))
    assert np.all(got[hit, 3:] == L) and np.all(got[~hit, 3:] == 0)


@pytest.mark.parametrize("bounce_tuning", [None, (128, 64, 0, 16), (256, 256, 0, 24), (256, 32, 1, 0, 4)])
def test_frame_graph_equals_eager(vx, cuda, bounce_tuning):
    import torch
    from vx_b200 import workloads as W
    wls, scenes, rays, begin, allr, d_rays, d_begin = _setup(vx, W, n=8, seed=14)
    n = allr.shape[0]
    batch = vx.Batch(scenes)
    if bounce_tuning is not None:
        batch.set_bounce_tuning(vx.BatchTuning(*bounce_tuning))
    bb = torch.from_numpy((2 * begin).astype(np.int32)).cuda()
    ph, bh = torch.zeros((n, 4), dtype=torch.int32, device="cuda"), torch.zeros((2 * n, 4), dtype=torch.int32,
                                                                               device="cuda")
    bounce = torch.zeros((2 * n, 6), dtype=torch.float32, device="cuda")
    # eager frame
    batch.cast(d_rays, d_begin, ph)
    vx.spawn_bounce_rays(d_rays, ph, 7, bounce)
    batch.cast(bounce, bb, bh)
    torch.cuda.synchronize()
    eager = (ph.cpu().numpy().copy(), bh.cpu().numpy().copy())
    ph.zero_(), bh.zero_(), bounce.zero_()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        batch.capture_frame(d_rays, d_begin, ph, bounce, bb, bh, 7, s.cuda_stream)
        batch.launch_frame(s.cuda_stream)
        batch.launch_frame(s.cuda_stream)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(ph.cpu().numpy(), eager[0])
    np.testing.assert_array_equal(bh.cpu().numpy(), eager[1])


@pytest.mark.parametrize("big,bounce_tuning", [(False, None), (False, (256, 256, 0, 24)), (True, (128, 64, 0, 16)),
                                                (True, (256, 32, 1, 0, 6))])
def test_compacted_frame_equals_eager(vx, cuda, big, bounce_tuning):
    """vx_batch_capture_frame_compact: primary and bounce hit records equal the eager frame's
    (whose bounce pass casts all 2n slots, zero-direction rays included); the compacted bounce
    rays are the eager bounce rays of the primary hits, per scene grouped by direction bin, then
    by chunk of 1024 primary rays, bounce k and primary order, the same on every launch.  `big` (more than 2^20 primary rays) gives
    scenes of many chunks with a partial last chunk."""
    import torch
    from vx_b200 import workloads as W
    if big:
        specs = W.config4_specs(4, seed=21, r_range=(6, 7.4), res_lo=(640, 480), res_hi=(1280, 720))
        wls = [W.build_spec(sp) for sp in specs]
        scenes = [vx.Scene(w.scene) for w in wls]
        rays = [w.rays(order="tiled") for w in wls]
        begin = np.concatenate([[0], np.cumsum([r.shape[0] for r in rays])]).astype(np.uint32)
        d_rays = torch.from_numpy(np.concatenate(rays).astype(np.float32)).cuda()
        d_begin = torch.from_numpy(begin.astype(np.int32)).cuda()
        assert d_rays.shape[0] > 1 << 20
    else:
        wls, scenes, rays, begin, allr, d_rays, d_begin = _setup(vx, W, n=8, seed=14)
    n = d_rays.shape[0]
    batch = vx.Batch(scenes)
    if bounce_tuning is not None:
        batch.set_bounce_tuning(vx.BatchTuning(*bounce_tuning))
    bb = torch.from_numpy((2 * begin.astype(np.int64)).astype(np.int32)).cuda()
    ph = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    bh = torch.zeros((2 * n, 4), dtype=torch.int32, device="cuda")
    bounce = torch.zeros((2 * n, 6), dtype=torch.float32, device="cuda")
    batch.cast(d_rays, d_begin, ph)
    vx.spawn_bounce_rays(d_rays, ph, 7, bounce)
    batch.set_tuning(*(bounce_tuning or (256, 32, 1, 0)))
    batch.cast(bounce, bb, bh)
    batch.set_tuning(256, 32, 1, 0)
    torch.cuda.synchronize()
    eager_ph, eager_bh, eager_bounce = ph.cpu().numpy().copy(), bh.cpu().numpy().copy(), bounce.cpu().numpy().copy()
    ph.fill_(-1), bh.fill_(-1), bounce.zero_()
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        batch.capture_frame_compact(d_rays, d_begin, ph, bounce, bh, 7, s.cuda_stream)
        batch.launch_frame(s.cuda_stream)
    torch.cuda.synchronize()
    first = bounce.cpu().numpy().copy()
    with torch.cuda.stream(s):
        bh.fill_(-1)
        bounce.zero_()
        batch.launch_frame(s.cuda_stream)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(ph.cpu().numpy(), eager_ph)
    np.testing.assert_array_equal(bh.cpu().numpy(), eager_bh)
    got = bounce.cpu().numpy()
    np.testing.assert_array_equal(got.view(np.uint32), first.view(np.uint32))
    hit = (eager_ph.view(vx.HIT_DTYPE).reshape(-1)["flags"] & 1).astype(bool)
    h = int(hit.sum())
    assert 0 < h < n
    # expected order: scene, direction bin, chunk of 1024 primary rays of the scene, k, primary ray
    pair = eager_bounce.reshape(n, 2, 6)
    scene = np.repeat(np.arange(len(begin) - 1), np.diff(begin.astype(np.int64)))
    idx = np.flatnonzero(hit)
    rows = pair[idx].reshape(-1, 6)
    sc = np.repeat(scene[idx], 2)
    prim = np.repeat(idx, 2)
    kk = np.tile(np.arange(2), idx.size)
    chunk = (prim - begin.astype(np.int64)[sc]) // 1024
    want = rows[np.lexsort((prim, kk, chunk, _direction_bin(rows), sc))]
    np.testing.assert_array_equal(got[:2 * h].view(np.uint32), want.view(np.uint32))
    # vx_batch_frame_compaction: per-scene ranges of the compacted rays and their hit slots
    sb, slot = batch.frame_compaction()
    assert sb[0] == 0 and sb[-1] == 2 * h and np.all(np.diff(sb.astype(np.int64)) >= 0)
    np.testing.assert_array_equal(np.diff(sb.astype(np.int64)), np.bincount(sc, minlength=len(begin) - 1))
    slots = np.flatnonzero(np.repeat(hit, 2))  # slot 2i + k of every bounce ray of a hit
    np.testing.assert_array_equal(np.sort(slot), slots)
    np.testing.assert_array_equal(got[:2 * h].view(np.uint32), eager_bounce[slot.astype(np.int64)].view(np.uint32))
    # vx_batch_launch_frame_host: the same frame from pinned host buffers
    rays_h = d_rays.cpu().pin_memory()
    ph_h = torch.full((n, 4), -1, dtype=torch.int32).pin_memory()
    bh_h = torch.full((2 * n, 4), -1, dtype=torch.int32).pin_memory()
    d_rays.zero_()  # the call copies the rays in itself
    torch.cuda.synchronize()  # the zeroing ran on another stream than the call's
    for _ in range(2):
        batch.launch_frame_host(rays_h, ph_h, bh_h, s.cuda_stream)
        np.testing.assert_array_equal(ph_h.numpy(), eager_ph)
        np.testing.assert_array_equal(bh_h.numpy(), eager_bh)
        ph_h.fill_(-1), bh_h.fill_(-1)


@pytest.mark.parametrize("parts", [1, 3, 7, 40])
def test_frame_in_parts_equals_whole_frame(vx, cuda, parts):
    """vx_batch_capture_frame_parts: pieces of consecutive primary rays (they begin and end
    inside scenes) give the whole compacted frame's primary and bounce records, replayed on the
    device and through vx_batch_launch_frame_host's pipelined copies; frame_compaction refuses
    a frame in parts."""
    import torch
    from vx_b200 import workloads as W
    wls, scenes, rays, begin, allr, d_rays, d_begin = _setup(vx, W, n=8, seed=31)
    n = d_rays.shape[0]
    batch = vx.Batch(scenes)
    batch.set_bounce_tuning(vx.BatchTuning(256, 32, 1, 0, 5))
    s = torch.cuda.Stream()
    ph = torch.full((n, 4), -1, dtype=torch.int32, device="cuda")
    bh = torch.full((2 * n, 4), -1, dtype=torch.int32, device="cuda")
    bounce = torch.zeros((2 * n, 6), dtype=torch.float32, device="cuda")
    with torch.cuda.stream(s):
        batch.capture_frame_compact(d_rays, d_begin, ph, bounce, bh, 9, s.cuda_stream)
        batch.launch_frame(s.cuda_stream)
    torch.cuda.synchronize()
    whole_ph, whole_bh = ph.cpu().numpy().copy(), bh.cpu().numpy().copy()
    ph.fill_(-1), bh.fill_(-1), bounce.zero_()
    torch.cuda.synchronize()
    with torch.cuda.stream(s):
        batch.capture_frame_parts(d_rays, d_begin, ph, bounce, bh, 9, parts, s.cuda_stream)
        batch.launch_frame(s.cuda_stream)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(ph.cpu().numpy(), whole_ph)
    np.testing.assert_array_equal(bh.cpu().numpy(), whole_bh)
    with pytest.raises(vx.VxError):
        batch.frame_compaction()
    rays_h = d_rays.cpu().pin_memory()
    ph_h = torch.full((n, 4), -1, dtype=torch.int32).pin_memory()
    bh_h = torch.full((2 * n, 4), -1, dtype=torch.int32).pin_memory()
    d_rays.zero_()  # the call copies the rays in itself
    torch.cuda.synchronize()
    for _ in range(2):
        batch.launch_frame_host(rays_h, ph_h, bh_h, s.cuda_stream)
        np.testing.assert_array_equal(ph_h.numpy(), whole_ph)
        np.testing.assert_array_equal(bh_h.numpy(), whole_bh)
        ph_h.fill_(-1), bh_h.fill_(-1)


def test_autotune_keeps_results(vx, cuda):
    import torch
    from vx_b200 import workloads as W
    wls, scenes, rays, begin, allr, d_rays, d_begin = _setup(vx, W, n=6, seed=15)
    plain = _plain(vx, scenes, rays, begin, d_rays)
    batch = vx.Batch(scenes)
    hits = torch.zeros_like(plain)
    t, ms = batch.autotune(d_rays, d_begin, hits)
    assert t.block in (128, 256) and t.rays_per_task % 32 == 0 and ms > 0
    hits.zero_()
    batch.cast(d_rays, d_begin, hits)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(hits.cpu().numpy(), plain.cpu().numpy())


def test_batch_rejects_bad_tuning(vx, cuda):
    from vx_b200 import workloads as W
    wl = W.config1(R=64, width=8, height=8)
    b = vx.Batch([vx.Scene(wl.scene)])
    with pytest.raises(vx.VxError):
        b.set_tuning(block=96)
    with pytest.raises(vx.VxError):
        b.set_tuning(rays_per_task=40)
    with pytest.raises(vx.VxError):
        b.set_tuning(refill=33)
    with pytest.raises(vx.VxError):
        b.set_tuning(refill=8, budget=24)  # a budget applies to static lanes only
    with pytest.raises(vx.VxError):
        b.set_tuning(budget=501)
    with pytest.raises(vx.VxError):
        b.set_bounce_tuning(vx.BatchTuning(256, 48, 1, 0))
    b.set_bounce_tuning(None)
