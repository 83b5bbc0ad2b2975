"""cfg3 urban scene with shadow rays (needs a B200), at 512^3 so the oracle
finishes in seconds: primary and shadow hits bit-exact vs the oracle; shadow
origins / directions equal their numpy restatement."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_urban_primary_and_shadow_rays_bit_exact(vx, vo, cuda):
    import torch
    from vx_b200 import workloads as W
    wl = W.config3(R=512, width=320, height=180, seed=3)
    s = vx.Scene(wl.scene)
    rays = wl.rays()
    n = rays.shape[0]
    d_rays = torch.from_numpy(rays).cuda()
    hits = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    col = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    s.cast_rays_dev(d_rays, hits, col)
    L = W.light_dir(3)
    shadow = torch.zeros((n, 6), dtype=torch.float32, device="cuda")
    vx.spawn_shadow_rays(d_rays, hits, L, shadow)
    sh = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    s.cast_rays_dev(shadow, sh)
    torch.cuda.synchronize()
    o = vo.OracleScene.from_dense(wl.bits, 512, wl.scene.max_levels)
    g = hits.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1)
    oh = o.cast_rays(rays)
    hit = (oh["flags"] & 1).astype(bool)
    assert hit.mean() > 0.2
    for f in ("brick", "node"):
        assert np.array_equal(g[f], oh[f]), f
    assert np.array_equal(g["flags"].astype(np.uint32), oh["flags"])
    assert np.array_equal(g["t"][hit].view(np.uint32), oh["t"][hit].view(np.uint32))
    want = W.bounce_rays_reference(rays, g, 0, vx.bounce_table())[0::2].copy()
    want[hit, 3:] = L
    got = shadow.cpu().numpy()
    np.testing.assert_array_equal(got[hit].view(np.uint32), want[hit].view(np.uint32))
    sg = sh.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1)
    so = o.cast_rays(got)
    assert np.array_equal(sg["flags"].astype(np.uint32), so["flags"])
    assert np.array_equal(sg["brick"], so["brick"]) and np.array_equal(sg["voxel"].astype(np.uint32), so["voxel"])
    sh_hit = (so["flags"] & 1).astype(bool)
    assert np.array_equal(sg["t"][sh_hit].view(np.uint32), so["t"][sh_hit].view(np.uint32))
