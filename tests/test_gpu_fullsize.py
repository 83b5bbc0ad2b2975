"""The benchmark frames at their full sizes against the CPU oracle (needs a B200).

The whole frame is cast on the GPU through the C ABI; a fixed stride of at
least 65,536 rays is then checked against the oracle on every field of the
hit record: flags, brick, node, voxel, scale, t (raw binary32 bits), the
reference traversal's work counters and the decoded DXT1 texel.

  cfg2  cave 1024^3 (depth 10), noise spacing 64, 5 octaves, 50 % fill, DXT1
        bricks, 1920x1080 primary rays.
  cfg3  urban 2048^3 (depth 11), 32x32 blocks, heights U[64,1800], DXT1
        bricks, 3840x2160 primary rays, then the compacted shadow pass
        (vx_cast_shadow_rays) toward the seeded light: the shadow record of
        every sampled ray is checked against the oracle's cast of the shadow
        ray built from the oracle's own primary hit.
"""
import numpy as np
import pytest

from test_gpu_parity import assert_hits_equal

pytestmark = pytest.mark.gpu

MIN_SAMPLE = 65536


def _stride(n):
    s = max(1, n // MIN_SAMPLE)
    while -(-n // s) < MIN_SAMPLE and s > 1:
        s -= 1
    return s


def _cast_full(vx, scene, rays_np):
    import torch
    n = rays_np.shape[0]
    rays = torch.from_numpy(rays_np).cuda()
    hits = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    col = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    cnt = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    scene.cast_rays_dev(rays, hits, col, cnt)
    return rays, hits, col, cnt


def _check_sample(vx, vo, o, brick_dxt, rays_np, hits, col, cnt, stride, label):
    idx = np.arange(0, rays_np.shape[0], stride)
    assert idx.size >= MIN_SAMPLE
    g = hits.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1)[idx]
    c = cnt.cpu().numpy().view(vx.COUNTER_DTYPE).reshape(-1)[idx]
    oh = o.cast_rays(rays_np[idx], threads=0)
    assert_hits_equal(g, oh, c, label)
    want = vo.hit_texels_dxt(brick_dxt, oh)
    np.testing.assert_array_equal(col.cpu().numpy()[idx].view(np.uint32), want.view(np.uint32))
    return idx, oh


def test_cfg2_cave1024_full_frame_sampled(vx, vo, cuda):
    import torch
    from vx_b200 import workloads as W
    bits = vx.synth_noise_dev(1024, 64, 5, 0.5, 2, False).cpu().numpy().view(np.uint64)
    wl = W.config2(R=1024, seed=2, bits=bits)
    scene = vx.Scene(wl.scene)
    rays_np = wl.rays(order="tiled")
    assert rays_np.shape[0] == 1920 * 1080
    _, hits, col, cnt = _cast_full(vx, scene, rays_np)
    torch.cuda.synchronize()
    o = vo.OracleScene.from_dense(bits, 1024, wl.scene.max_levels)
    idx, oh = _check_sample(vx, vo, o, wl.scene.brick_color, rays_np, hits, col, cnt, _stride(rays_np.shape[0]),
                            wl.name)
    assert (oh["flags"] & 1).mean() > 0.3
    assert np.count_nonzero(oh["flags"] & vx.VX_RAY_ITER_CAP) > 0  # capped rays are part of the sample


def test_cfg3_urban2048_full_frame_and_shadow_pass_sampled(vx, vo, cuda):
    import torch
    from vx_b200 import workloads as W
    wl = W.config3()
    assert (wl.R, wl.width, wl.height) == (2048, 3840, 2160)
    scene = vx.Scene(wl.scene)
    rays_np = wl.rays(order="tiled")
    n = rays_np.shape[0]
    rays, hits, col, cnt = _cast_full(vx, scene, rays_np)
    L = W.light_dir(3)
    sh = torch.full((n, 4), -1, dtype=torch.int32, device="cuda")
    scene.cast_shadow_rays_dev(rays, hits, L, sh)
    torch.cuda.synchronize()
    o = vo.OracleScene.from_dense(wl.bits, 2048, wl.scene.max_levels)
    idx, oh = _check_sample(vx, vo, o, wl.scene.brick_color, rays_np, hits, col, cnt, _stride(n), wl.name)
    hit = (oh["flags"] & 1).astype(bool)
    assert 0.2 < hit.mean() < 0.95
    # shadow rays of the oracle's own hits: origin = hit point + 1e-3 * normal, direction = light
    srays = W.bounce_rays_reference(rays_np[idx], oh, 0, vx.bounce_table())[0::2].copy()
    srays[hit, 3:] = L
    srays[~hit, 3:] = 0.0
    so = o.cast_rays(srays, threads=0)
    sg = sh.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1)[idx]
    assert_hits_equal(sg, so, None, wl.name + " shadow")
    assert np.all(so["flags"][~hit] & vx.VX_RAY_INVALID)
    shadowed = (so["flags"][hit] & 1).mean()
    assert 0.05 < shadowed < 0.95
