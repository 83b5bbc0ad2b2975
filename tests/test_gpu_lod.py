"""castRayWithLOD on the GPU (vx_cast_rays_lod / vx_cast_rays_host_lod) against
the oracle, bit for bit (needs a B200).  LOD hits must carry the oracle's
distance bits, cell scale, parent descriptor and iteration counts; rays that
reach full detail must equal castRay's results."""
import math

import numpy as np
import pytest

from test_gpu_parity import assert_hits_equal, gpu_cast, scene_from_oracle

pytestmark = pytest.mark.gpu

FLT_MAX = 3.4028234663852886e38


def gpu_cast_lod(vx, scene, rays, lod, tmin=0.0, tmax=FLT_MAX):
    import torch
    s = scene if isinstance(scene, vx.Scene) else vx.Scene(scene)
    n = rays.shape[0]
    r = torch.from_numpy(np.ascontiguousarray(rays, np.float32)).cuda()
    hits = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    cw = s.color_width()
    color = None
    if cw:
        color = torch.full((n, cw), 7, dtype=torch.int32 if cw == 1 else torch.float32, device="cuda")
    counters = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    s.cast_rays_dev(r, hits, color, counters, tmin, tmax, lod=lod)
    torch.cuda.synchronize()
    h = hits.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1)
    c = None if color is None else color.cpu().numpy()
    return h, c, counters.cpu().numpy().view(vx.COUNTER_DTYPE).reshape(-1)


LODS = [(0.0, 0.005), (0.0, 0.02), (0.0, 0.1), (0.25, 0.03), (0.0, 1.0)]


@pytest.mark.parametrize("lod", LODS)
def test_lod_noise_rgba8_bit_exact(vx, vo, cuda, lod):
    from vx_b200 import workloads as W
    wl = W.config1(R=128, width=96, height=96, seed=21)
    o = vo.OracleScene.from_dense(wl.bits, 128, wl.scene.max_levels)
    rays = np.concatenate([wl.rays(), W.random_rays(12000, 128, seed=22)])
    g, col, cnt = gpu_cast_lod(vx, wl.scene, rays, lod)
    oh = o.cast_rays_lod(rays, lod)
    assert_hits_equal(g, oh, cnt, f"lod {lod}")
    is_lod = ((oh["flags"] & 1) == 1) & (oh["brick"] == 0xFFFFFFFF)
    assert is_lod.any()
    assert np.all(col[is_lod] == 0)  # no voxel, no colour
    hit = ((oh["flags"] & 1) == 1) & ~is_lod
    want = wl.scene.brick_color[oh["brick"][hit].astype(np.int64) * 512 + oh["voxel"][hit]]
    np.testing.assert_array_equal(col[hit, 0].view(np.uint32), want)


def test_lod_dxt_scene_and_screen_space_params(vx, vo, cuda):
    from vx_b200 import workloads as W
    wl = W.config2(R=128, width=160, height=90, seed=23)
    o = vo.OracleScene.from_dense(wl.bits, 128, wl.scene.max_levels)
    rays = np.concatenate([wl.rays(), W.random_rays(10000, 128, seed=24)])
    s = vx.Scene(wl.scene)
    base = vx.lod_from_camera(math.radians(70.0), 90)
    for bias in (0.0, 2.0, 4.0):
        lod = vx.lod_with_bias(base, bias).as_tuple()
        g, col, cnt = gpu_cast_lod(vx, s, rays, lod)
        oh = o.cast_rays_lod(rays, lod)
        assert_hits_equal(g, oh, cnt, f"bias {bias}")
        is_lod = ((oh["flags"] & 1) == 1) & (oh["brick"] == 0xFFFFFFFF)
        assert np.all(col[is_lod] == 0)


@pytest.mark.parametrize("lod", [(0.0, 0.0), (0.5, 0.0), (0.0, -0.25)])
def test_disabled_lod_equals_cast_rays(vx, cuda, lod):
    from vx_b200 import workloads as W
    wl = W.config1(R=64, width=64, height=64, seed=25)
    s = vx.Scene(wl.scene)
    rays = np.concatenate([wl.rays(), W.random_rays(4000, 64, seed=26)])
    a, ca, na = gpu_cast_lod(vx, s, rays, lod)
    b, cb, nb = gpu_cast(vx, s, rays)
    assert a.tobytes() == b.tobytes() and na.tobytes() == nb.tobytes()
    np.testing.assert_array_equal(ca, cb)


def test_lod_host_entry_matches_device(vx, cuda):
    from vx_b200 import workloads as W
    wl = W.config2(R=64, width=64, height=48, seed=27)
    s = vx.Scene(wl.scene)
    rays = wl.rays()
    lod = (0.1, 0.05)
    gd, cd, _ = gpu_cast_lod(vx, s, rays, lod)
    gh, ch = s.cast_rays_host(rays, lod=lod)
    np.testing.assert_array_equal(gd.view(np.uint8), gh.view(np.uint8))
    np.testing.assert_array_equal(cd.view(np.uint32), ch.view(np.uint32))


def test_reference_lod_cases_through_facade(vx, vo, cuda):
    """The LODRayCastingTest scenes (SVO/tests/test_lod.cpp:158-330) through the
    castRay-shaped facade, equal to the oracle's castRay*LOD."""
    for pos, wmax, depth, origin, fov, height in [((50, 50, 50), 100, 8, (50, 50, 500), 60.0, 600),
                                                   ((5, 5, 5), 10, 6, (5, 5, 8), 60.0, 1080),
                                                   ((5, 5, 5), 10, 6, (5, 5, 15), 60.0, 1080)]:
        o = vo.OracleScene.from_positions([pos], (0, 0, 0), (wmax,) * 3, depth)
        oct_ = vx.CudaOctree(vx.Scene(scene_from_oracle(vx, o, ((0, 0, 0), (wmax,) * 3), depth)))
        fovr = math.radians(fov)
        a = oct_.castRayScreenSpaceLOD(origin, (0, 0, -1), fovr, height)
        b = o.castRayScreenSpaceLOD(origin, (0, 0, -1), fovr, height)
        assert a.hit == bool(b["flags"] & 1)
        if a.hit:
            assert np.float32(a.tMin).view(np.uint32) == b["t"].view(np.uint32) and a.scale == b["scale"]
        for lod in [(0.0, 0.01), (0.0, 0.0)]:
            a = oct_.castRayWithLOD(origin, (0, 0, -1), lod)
            b = o.castRayWithLOD(origin, (0, 0, -1), lod)
            assert a.hit == bool(b["flags"] & 1)
        a, b = oct_.castRayLOD(origin, (0, 0, -1), 0.0), oct_.castRay(origin, (0, 0, -1))
        assert a == b


def test_lod_full_size_cfg1(vx, vo, cuda):
    """256^3 noise, 512x512 primary rays, LOD parameters of a 60-degree camera
    at 512 rows biased coarser by 2^6 so that cuts happen inside the world."""
    from vx_b200 import workloads as W
    wl = W.config1()
    o = vo.OracleScene.from_dense(wl.bits, 256, 8)
    rays = wl.rays()
    lod = vx.lod_with_bias(vx.lod_from_camera(math.radians(60.0), 512), 6.0).as_tuple()
    g, _, cnt = gpu_cast_lod(vx, wl.scene, rays, lod)
    oh = o.cast_rays_lod(rays, lod)
    assert_hits_equal(g, oh, cnt, "cfg1 lod")
    assert (((oh["flags"] & 1) == 1) & (oh["brick"] == 0xFFFFFFFF)).mean() > 0.05
