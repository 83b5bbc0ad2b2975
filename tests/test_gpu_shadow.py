"""vx_cast_shadow_rays (needs a B200): the compacted shadow pass writes, for
every primary ray, exactly what spawning the shadow rays of all slots and
casting them all writes, including the invalid record of primary misses."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _frame(vx, W, wl, L, t_max):
    import torch
    s = vx.Scene(wl.scene)
    rays = torch.from_numpy(wl.rays(order="tiled")).cuda()
    n = rays.shape[0]
    hits = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    s.cast_rays_dev(rays, hits)
    shadow = torch.zeros((n, 6), dtype=torch.float32, device="cuda")
    vx.spawn_shadow_rays(rays, hits, L, shadow)
    want = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    s.cast_rays_dev(shadow, want, t_max=t_max)
    torch.cuda.synchronize()
    return s, rays, hits, want.cpu().numpy()


@pytest.mark.parametrize("kind,t_max", [("urban", None), ("cave", None), ("cave", 40.0)])
def test_shadow_pass_equals_spawn_then_cast(vx, cuda, kind, t_max):
    import torch
    from vx_b200 import workloads as W
    # 257 x 131 primary rays: not a multiple of the 1,024-ray compaction chunk
    wl = W.config3(R=256) if kind == "urban" else W.config2(R=128, width=257, height=131, seed=41)
    L = W.light_dir(3)
    tm = vx.FLT_MAX if t_max is None else t_max
    s, rays, hits, want = _frame(vx, W, wl, L, tm)
    n = rays.shape[0]
    flags = want.view(vx.HIT_DTYPE).reshape(-1)["flags"]
    primary = (hits.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1)["flags"] & 1).astype(bool)
    assert 0 < primary.sum() < n and np.any(flags & 1)
    got = torch.full((n, 4), -1, dtype=torch.int32, device="cuda")
    for _ in range(2):  # the scratch keeps the last call's contents
        got.fill_(-1)
        s.cast_shadow_rays_dev(rays, hits, L, got, t_max=tm)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(got.cpu().numpy(), want)


def test_shadow_pass_rejects_bad_arguments(vx, cuda):
    import torch
    from vx_b200 import workloads as W
    wl = W.config1(R=64, width=8, height=8, seed=3)
    s = vx.Scene(wl.scene)
    rays = torch.zeros((64, 6), dtype=torch.float32, device="cuda")
    hits = torch.zeros((64, 4), dtype=torch.int32, device="cuda")
    with pytest.raises(vx.VxError):
        s.cast_shadow_rays_dev(rays, hits, [0.0, 1.0, 0.0], hits[:, :3].contiguous().view(-1)[1:])
