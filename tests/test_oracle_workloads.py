"""The oracle-side workload builders (oracle/workloads_ref.py, oracle/vx_oracle_synth.cpp)
produce the product's inputs bit for bit, so the CPU baseline and the reference arm of the
benchmark can build the frames without loading libvx.so.  CPU only."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def wr(vo):
    import workloads_ref
    return workloads_ref


def _pc_words(pc):
    return np.frombuffer(bytes(memoryview(pc)), dtype=np.uint32)


@pytest.mark.parametrize("R,spacing,octaves,fill,seed,shell", [
    (64, 8, 3, 0.1, 1, True), (64, 16, 3, 0.5, 2, False), (128, 32, 4, 0.3, 5, False),
    (128, 4, 3, 0.9, 7, False), (64, 8, 3, 0.0, 3, True), (64, 8, 3, 1.0, 4, False)])
def test_noise_bits_equal_product(vx, wr, R, spacing, octaves, fill, seed, shell):
    want = vx.synth_noise(R, spacing, octaves, fill, seed, shell)
    got = wr.noise_bits(R, spacing, octaves, fill, seed, shell)
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("R,hmin,hmax,seed", [(64, 2, 56, 1), (128, 4, 112, 9), (256, 8, 225, 3)])
def test_urban_bits_equal_product(vx, wr, R, hmin, hmax, seed):
    np.testing.assert_array_equal(wr.urban_bits(R, hmin, hmax, seed), vx.synth_urban(R, hmin, hmax, seed))


def test_bounce_table_equals_product(vx, wr):
    np.testing.assert_array_equal(wr.bounce_table().view(np.uint32), vx.bounce_table().view(np.uint32))


def test_cameras_and_specs_equal_product(vx, wr):
    from vx_b200 import workloads as W
    bits = vx.synth_noise(128, 8, 3, 0.5, 11, False)
    for seed in (1, 2, 40):
        np.testing.assert_array_equal(wr.empty_voxel_camera(bits, 128, seed, 70.0, 640, 360).view(np.uint32),
                                      _pc_words(W.empty_voxel_camera(bits, 128, seed, 70.0, 640, 360)))
    np.testing.assert_array_equal(wr.look_camera([1024.0, 1843.2, -512.0], [0.05, -0.45, 1.0], 60.0, 3840,
                                                 2160).view(np.uint32),
                                  _pc_words(W.look_camera([1024.0, 1843.2, -512.0], [0.05, -0.45, 1.0], 60.0,
                                                          3840, 2160)))
    for a, b in zip(wr.cfg4_specs(64, seed=4), W.config4_specs(64, seed=4)):
        assert (a.R, a.kind, a.fill, a.color, a.width, a.height, a.seed) == \
            (b.R, b.kind, b.fill, b.color, b.width, b.height, b.seed)
    np.testing.assert_array_equal(wr.tile_order(1920, 1080), W.tile_order(1920, 1080))
    np.testing.assert_array_equal(wr.light_dir(3).view(np.uint32), W.light_dir(3).view(np.uint32))


def test_frames_equal_product(vx, wr):
    """Small instances of the cave, urban and batched frames: bits and primary rays."""
    from vx_b200 import workloads as W
    a, b = wr.cfg2(R=128, width=96, height=64, seed=5), W.config2(R=128, width=96, height=64, seed=5)
    np.testing.assert_array_equal(a.bits, b.bits)
    np.testing.assert_array_equal(a.rays().view(np.uint32), b.rays(order="tiled").view(np.uint32))
    a, b = wr.cfg3(R=256, width=64, height=48), W.config3(R=256, width=64, height=48)
    np.testing.assert_array_equal(a.bits, b.bits)
    np.testing.assert_array_equal(a.rays().view(np.uint32), b.rays(order="tiled").view(np.uint32))
    specs = wr.cfg4_specs(6, seed=21, r_range=(6, 7.4), res_lo=(48, 40), res_hi=(160, 96))
    wspecs = W.config4_specs(6, seed=21, r_range=(6, 7.4), res_lo=(48, 40), res_hi=(160, 96))
    for sa, sb in zip(specs, wspecs):
        fa, fb = wr.cfg4_frame(sa), W.build_spec(sb)
        np.testing.assert_array_equal(fa.bits, fb.bits)
        np.testing.assert_array_equal(fa.rays().view(np.uint32), fb.rays(order="tiled").view(np.uint32))


def test_secondary_rays_equal_numpy_restatement(vx, vo, wr):
    """Bounce and shadow rays from the oracle's own hit records equal the product's definition
    as restated in numpy (workloads.bounce_rays_reference), for a frame index offset too."""
    from vx_b200 import workloads as W
    wl = W.config1(R=64, width=48, height=32, seed=4)
    o = vo.OracleScene.from_dense(wl.bits, 64, wl.scene.max_levels)
    rays = wl.rays()
    oh = o.cast_rays(rays)
    assert (oh["flags"] & 1).mean() > 0.2
    want = W.bounce_rays_reference(rays, oh, 77, vx.bounce_table())
    np.testing.assert_array_equal(wr.spawn_bounce(rays, oh, 77).view(np.uint32), want.view(np.uint32))
    # rays [100, 300) of the frame, passed with their frame positions
    idx = np.arange(100, 300, dtype=np.uint64)
    np.testing.assert_array_equal(wr.spawn_bounce(rays[100:300], oh[100:300], 77, idx).view(np.uint32),
                                  want[200:600].view(np.uint32))
    L = W.light_dir(3)
    sh = W.bounce_rays_reference(rays, oh, 0, vx.bounce_table())[0::2].copy()
    hit = (oh["flags"] & 1).astype(bool)
    sh[hit, 3:] = L
    np.testing.assert_array_equal(wr.spawn_shadow(rays, oh, L).view(np.uint32), sh.view(np.uint32))
