"""Device scene builder (vx_scene_create_dense_dev) against the host builder
(vx_build_dense, itself pinned to the oracle's restated rebuild): every array
identical, colour and normal payloads included (needs a B200)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bits_with(R, voxels):
    bits = np.zeros(R * R * (R // 64), np.uint64)
    for x, y, z in voxels:
        w = (z * R + y) * (R // 64) + x // 64
        bits[w] |= np.uint64(1) << np.uint64(x % 64)
    return bits


def _device_scene(vx, bits, R, levels, color_kind=0, seed=0, normals=False):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(bits).view(np.int64)).cuda()
    return vx.scene_from_dense_dev(t, R, levels, color_kind, seed, normals)


def _assert_same(vx, got, bits, R, levels, color_kind=0, seed=0, normals=False):
    want = vx.build_dense(bits, R, levels)
    for k in ["nodes", "node_brick", "grid_lookup", "brick_coord", "brick_occ"]:
        np.testing.assert_array_equal(getattr(got, k), getattr(want, k), err_msg=k)
    assert got.world_min == want.world_min and got.world_max == want.world_max
    assert got.max_levels == want.max_levels and got.bricks_per_axis == want.bricks_per_axis
    if color_kind == vx.VX_COLOR_RGBA8:
        np.testing.assert_array_equal(got.brick_color, vx.synth_rgba8(want.brick_coord, seed))
    elif color_kind == vx.VX_COLOR_DXT1:
        np.testing.assert_array_equal(got.brick_color, vx.synth_dxt1(want.brick_coord, seed))
    else:
        assert got.brick_color is None
    if normals and want.brick_count:
        np.testing.assert_array_equal(got.brick_normal, vx.build_normals(want.brick_occ.reshape(-1, 16)))
    return want


@pytest.mark.parametrize("R,fill,seed", [(64, 0.1, 1), (64, 0.5, 2), (128, 0.3, 3), (192, 0.2, 4), (256, 0.1, 5)])
def test_noise_scenes_identical(vx, cuda, R, fill, seed):
    levels = int(np.ceil(np.log2(R)))
    bits = vx.synth_noise(R, max(4, R // 16), 3, fill, seed, seed % 2 == 1)
    s = _device_scene(vx, bits, R, levels, vx.VX_COLOR_RGBA8 if seed % 2 else vx.VX_COLOR_DXT1, seed, True)
    _assert_same(vx, s.arrays, bits, R, levels, s.color_kind, seed, True)


def test_urban_scene_identical(vx, cuda):
    R = 256
    bits = vx.synth_urban(R, 8, 220, 9)
    s = _device_scene(vx, bits, R, 8, vx.VX_COLOR_DXT1, 9, True)
    _assert_same(vx, s.arrays, bits, R, 8, vx.VX_COLOR_DXT1, 9, True)


@pytest.mark.parametrize("voxels", [[(0, 0, 0)], [(3, 5, 7), (9, 1, 2)], [(63, 63, 63)], [(100, 3, 3)],
                                    [(0, 0, 0), (127, 127, 127)], [(17, 40, 33)]])
def test_sparse_scenes_identical(vx, cuda, voxels):
    """Single bricks, bricks in the first octant only (the tree stops climbing
    at the first single node at coordinate 0) and opposite corners."""
    R = 128
    bits = _bits_with(R, voxels)
    for levels in (7, 9):
        s = _device_scene(vx, bits, R, levels)
        want = _assert_same(vx, s.arrays, bits, R, levels)
        assert s.info().node_count == want.node_count


def test_empty_scene(vx, cuda):
    bits = np.zeros(64 * 64, np.uint64)
    s = _device_scene(vx, bits, 64, 6, vx.VX_COLOR_RGBA8, 1, True)
    i = s.info()
    assert i.node_count == 0 and i.brick_count == 0 and not i.has_normals
    assert np.all(s.arrays.grid_lookup == 0xFFFFFFFF)


def test_too_few_levels_rejected(vx, cuda):
    bits = _bits_with(128, [(0, 0, 0), (127, 127, 127)])
    with pytest.raises(vx.VxError):
        vx.build_dense(bits, 128, 5)
    with pytest.raises(vx.VxError):
        _device_scene(vx, bits, 128, 5)


def test_cfg2_scale_identical_and_casts_equal(vx, cuda):
    """1024^3, 50 % noise: the device-built scene equals the host build and
    casts the same hits."""
    import torch
    from vx_b200 import workloads as W
    R = 1024
    bits_t = vx.synth_noise_dev(R, 64, 5, 0.5, 2, False)
    bits = bits_t.cpu().numpy().view(np.uint64)
    s = vx.scene_from_dense_dev(bits_t, R, 10, vx.VX_COLOR_DXT1, 2 ^ 0xD7C1)
    got = s.arrays
    want = _assert_same(vx, got, bits, R, 10, vx.VX_COLOR_DXT1, 2 ^ 0xD7C1)
    rays = torch.from_numpy(W.random_rays(200000, R, seed=5)).cuda()
    h1 = torch.zeros((rays.shape[0], 4), dtype=torch.int32, device="cuda")
    h2 = torch.zeros_like(h1)
    s.cast_rays_dev(rays, h1)
    want.color_kind, want.brick_color = got.color_kind, got.brick_color
    vx.Scene(want).cast_rays_dev(rays, h2)
    torch.cuda.synchronize()
    assert torch.equal(h1, h2)


def test_scene_save_load_round_trip(vx, cuda, tmp_path):
    """A device-built scene saved to a VXSC file and loaded back casts the same
    hits and holds the same arrays."""
    import torch
    from vx_b200 import workloads as W
    R = 256
    bits = vx.synth_noise(R, 32, 4, 0.2, 6, True)
    s = _device_scene(vx, bits, R, 8, vx.VX_COLOR_DXT1, 3, True)
    p = str(tmp_path / "scene.vxsc")
    s.save(p)
    t = vx.Scene.load(p)
    a, b = s.arrays, t.arrays
    for k in ["nodes", "node_brick", "grid_lookup", "brick_coord", "brick_occ", "brick_color", "brick_normal"]:
        np.testing.assert_array_equal(getattr(a, k), getattr(b, k), err_msg=k)
    rays = torch.from_numpy(W.random_rays(50000, R, seed=8)).cuda()
    h1 = torch.zeros((rays.shape[0], 4), dtype=torch.int32, device="cuda")
    h2 = torch.zeros_like(h1)
    s.cast_rays_dev(rays, h1)
    t.cast_rays_dev(rays, h2)
    torch.cuda.synchronize()
    assert torch.equal(h1, h2)
