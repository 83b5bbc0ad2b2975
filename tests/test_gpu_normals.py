"""DXT normal payload and compressed shading on the GPU (needs a B200): the
device builder (vx_build_normals_dev) equals the oracle's restatement of the
rebuild's normal compression bit for bit, vx_hit_normals equals the oracle's
decode per hit, and vx_render with a normal payload equals the oracle's
compressed shading per pixel."""
import numpy as np
import pytest

from test_gpu_parity import assert_hits_equal
from test_normals import _bricks, _shaped_bricks

pytestmark = pytest.mark.gpu


def _dev_normals(vx, occ):
    import torch
    o = torch.from_numpy(np.ascontiguousarray(occ, np.uint32).view(np.int32).reshape(-1)).cuda()
    out = torch.zeros(occ.shape[0] * 64, dtype=torch.int64, device="cuda")
    vx.build_normals_dev(o, out)
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint64).reshape(-1, 32, 2)


def test_device_builder_equals_oracle_random_bricks(vx, vo, cuda):
    occ = _bricks(7, 3000)
    np.testing.assert_array_equal(_dev_normals(vx, occ), vo.brick_normals(occ))


def test_device_builder_equals_oracle_shaped_bricks(vx, vo, cuda):
    occ = _shaped_bricks(8, 1500)
    np.testing.assert_array_equal(_dev_normals(vx, occ), vo.brick_normals(occ))


@pytest.mark.parametrize("R", [128, 256])
def test_device_builder_equals_oracle_noise_scene(vx, vo, cuda, R):
    from vx_b200 import workloads as W
    wl = W.config1(R=R, width=8, height=8, seed=32)
    occ = wl.scene.brick_occ.reshape(-1, 16)
    got = _dev_normals(vx, occ)
    np.testing.assert_array_equal(got, vo.brick_normals(occ))
    np.testing.assert_array_equal(got, vx.build_normals(occ))


def _scene_with_normals(vx, wl):
    import dataclasses
    a = dataclasses.replace(wl.scene, brick_normal=vx.build_normals(wl.scene.brick_occ.reshape(-1, 16)))
    return a, vx.Scene(a)


def test_hit_normals_equal_oracle(vx, vo, cuda):
    import torch
    from vx_b200 import workloads as W
    wl = W.config2(R=128, width=120, height=80, seed=33)
    a, s = _scene_with_normals(vx, wl)
    rays = np.concatenate([wl.rays(), W.random_rays(6000, 128, seed=34)])
    n = rays.shape[0]
    r = torch.from_numpy(rays).cuda()
    hits = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    s.cast_rays_dev(r, hits)
    nrm = torch.full((n, 3), 7.0, dtype=torch.float32, device="cuda")
    s.hit_normals_dev(hits, nrm)
    torch.cuda.synchronize()
    g = hits.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1)
    got = nrm.cpu().numpy()
    hit = np.flatnonzero(g["flags"] & 1)
    assert hit.size > 1000
    for i in hit:
        want = vo.hit_normal_dxt(a.brick_normal, int(g["brick"][i]), int(g["voxel"][i]))
        np.testing.assert_array_equal(got[i].view(np.uint32), want.view(np.uint32))
    assert np.all(got[(g["flags"] & 1) == 0] == 0)


def test_hit_normals_needs_payload(vx, cuda):
    import torch
    from vx_b200 import workloads as W
    wl = W.config1(R=64, width=8, height=8, seed=35)
    s = vx.Scene(wl.scene)
    hits = torch.zeros((4, 4), dtype=torch.int32, device="cuda")
    out = torch.zeros((4, 3), dtype=torch.float32, device="cuda")
    with pytest.raises(vx.VxError):
        s.hit_normals_dev(hits, out)


@pytest.mark.parametrize("kind", ["rgba8", "dxt1"])
def test_render_with_normals_matches_oracle_shading(vx, vo, cuda, kind):
    import torch
    from vx_b200 import workloads as W
    wl = W.config1(R=128, width=96, height=80, seed=36) if kind == "rgba8" else W.config2(R=128, width=96,
                                                                                          height=80, seed=37)
    a, s = _scene_with_normals(vx, wl)
    n = wl.width * wl.height
    img = torch.zeros(n, dtype=torch.int32, device="cuda")
    hits = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    s.render_dev(wl.camera, wl.width, wl.height, img, hits)
    torch.cuda.synchronize()
    g = hits.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1)
    image = img.cpu().numpy().view(np.uint32)
    o = vo.OracleScene.from_dense(wl.bits, 128, wl.scene.max_levels)
    oh = o.cast_rays(wl.rays())
    assert_hits_equal(g, oh, None, "render hits")
    for i in range(n):
        hit = bool(oh["flags"][i] & 1)
        nd = np.zeros(3, np.float32)
        col = np.zeros(3, np.float32)
        if hit:
            b, v = int(oh["brick"][i]), int(oh["voxel"][i])
            nd = vo.hit_normal_dxt(a.brick_normal, b, v)
            if kind == "rgba8":
                c = int(a.brick_color[b * 512 + v])
                col = np.array([c & 255, (c >> 8) & 255, (c >> 16) & 255], np.float32) / np.float32(255.0)
            else:
                col = vo.hit_texel_dxt(a.brick_color, b, v)
        uv_y = (np.float32(i // wl.width) + np.float32(0.5)) / np.float32(wl.height)
        want = vo.shade_dxt_normal(col, hit, nd, (int(oh["flags"][i]) >> 1) & 3, bool(oh["flags"][i] & 8),
                                   float(uv_y))
        assert image[i] == want, (i, hex(image[i]), hex(want))


def test_device_dxt1_builder_equals_oracle(vx, vo, cuda):
    import torch
    from test_normals import _colours
    occ = _bricks(16, 2000)
    rgb = _colours(17, 2000)
    o = torch.from_numpy(occ.view(np.int32).reshape(-1)).cuda()
    c = torch.from_numpy(rgb.reshape(-1)).cuda()
    out = torch.zeros(2000 * 32, dtype=torch.int64, device="cuda")
    vx.build_dxt1_dev(c, o, out)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint64), vo.brick_dxt1(rgb, occ))
