"""Screen-space LOD cut on the CPU: LODParameters (SVO/include/SVOLOD.h:50-177)
and castRayWithLOD (SVO/src/SVOTraversal.cpp:198-232, :613-651) in the oracle,
ported from the reference's SVO/tests/test_lod.cpp and test_octree_queries.cpp,
plus the product's host-side parameter helpers (vx_lod_from_camera /
vx_lod_with_bias), which need no GPU."""
import math

import numpy as np
import pytest

FOV60, FOV90 = math.radians(60.0), math.radians(90.0)


def _proj(lod, d):
    """LODParameters::getProjectedPixelSize in binary32."""
    return np.float32(np.float32(d) * np.float32(lod[1])) + np.float32(lod[0])


# -- LODParametersTest (test_lod.cpp:41-153) --------------------------------------------

def test_default_disables_lod(vx):
    p = vx.LodParams()
    assert p.ray_orig_size == 0.0 and p.ray_dir_size == 0.0


def test_from_camera_valid_and_equal_to_oracle(vx, vo):
    for fov in (FOV60, FOV90, 1.2):
        for h in (600, 720, 1080, 2160):
            p = vx.lod_from_camera(fov, h)
            o = vo.lod_from_camera(fov, h)
            assert p.ray_orig_size == 0.0 and p.ray_dir_size > 0.0
            assert np.float32(p.ray_dir_size).view(np.uint32) == np.float32(o[1]).view(np.uint32)


def test_cone_spread_orders(vx):
    assert vx.lod_from_camera(FOV60, 1080).ray_dir_size < vx.lod_from_camera(FOV60, 720).ray_dir_size
    assert vx.lod_from_camera(FOV90, 720).ray_dir_size > vx.lod_from_camera(FOV60, 720).ray_dir_size


def test_projected_size_and_termination(vx):
    p = vx.lod_from_camera(FOV60, 720).as_tuple()
    s1, s10, s100 = _proj(p, 1.0), _proj(p, 10.0), _proj(p, 100.0)
    assert s10 > s1 and s100 > s10 and abs(s10 / s1 - 10.0) < 0.01
    assert _proj(p, 100.0) >= np.float32(0.01)  # ShouldTerminateAtLargeDistance
    assert not _proj(p, 0.1) >= np.float32(1.0)  # ShouldNotTerminateNearby


def test_bias_and_near_plane_equal_to_oracle(vx, vo):
    base = vx.lod_from_camera(FOV60, 720)
    for bias in (-2.0, -1.0, 0.0, 0.5, 1.0, 3.0):
        p = vx.lod_with_bias(base, bias).as_tuple()
        o = vo.lod_with_bias(base.as_tuple(), bias)
        np.testing.assert_array_equal(np.float32(p).view(np.uint32), np.float32(o).view(np.uint32))
    coarser, finer = vx.lod_with_bias(base, 1.0).as_tuple(), vx.lod_with_bias(base, -1.0).as_tuple()
    assert _proj(coarser, 10.0) > _proj(base.as_tuple(), 10.0) > _proj(finer, 10.0)
    near = vx.lod_from_camera(FOV60, 720, 0.1)
    assert near.ray_orig_size > 0.0 and near.ray_dir_size == base.ray_dir_size
    o = vo.lod_from_camera(FOV60, 720, 0.1)
    assert np.float32(near.ray_orig_size).view(np.uint32) == np.float32(o[0]).view(np.uint32)


def test_bad_screen_height_rejected(vx):
    with pytest.raises(vx.VxError):
        vx.lod_from_camera(FOV60, 0)


# -- esvoScaleToWorldSize (test_lod.cpp ESVOScaleHelperTest) ---------------------------

def test_esvo_scale_to_world_size():
    size = lambda sc, w: float(np.ldexp(np.float32(1.0), sc - 23) * np.float32(w))
    assert abs(size(22, 100.0) - 50.0) < 1.0
    assert size(10, 100.0) < size(22, 100.0) and size(0, 100.0) < 0.1


# -- LODRayCastingTest (test_lod.cpp:158-330) and CastRayLODZeroBias
#    (test_octree_queries.cpp:209-220) on the oracle ----------------------------------

def test_distant_voxel_terminates_early(vo):
    s = vo.OracleScene.from_positions([(50, 50, 50)], (0, 0, 0), (100, 100, 100), 8)
    lod = s.castRayScreenSpaceLOD((50, 50, 500), (0, 0, -1), FOV60, 600)
    full = s.castRay((50, 50, 500), (0, 0, -1))
    if (lod["flags"] & 1) and (full["flags"] & 1):
        assert lod["scale"] <= full["scale"]


def test_nearby_voxel_reaches_full_detail(vo):
    s = vo.OracleScene.from_positions([(5, 5, 5)], (0, 0, 0), (10, 10, 10), 6)
    lod = s.castRayScreenSpaceLOD((5, 5, 8), (0, 0, -1), FOV60, 1080)
    full = s.castRay((5, 5, 8), (0, 0, -1))
    if (lod["flags"] & 1) and (full["flags"] & 1):
        assert lod["scale"] >= full["scale"] - 1


@pytest.mark.parametrize("lod", [(0.0, 0.0), (0.0, -1.0)])
def test_disabled_lod_matches_regular_cast(vo, lod):
    s = vo.OracleScene.from_positions([(5, 5, 5)], (0, 0, 0), (10, 10, 10), 6)
    for o, d in [((5, 5, 15), (0, 0, -1)), ((5.5, 5.5, -3), (0, 0, 1)), ((-1, 5.5, 5.5), (1, 0.01, 0))]:
        a = s.castRayWithLOD(o, d, lod)
        b = s.castRay(o, d)
        assert a.tobytes() == b.tobytes()
    a = s.castRayLOD((5, 5, 15), (0, 0, -1), 0.0)
    assert a.tobytes() == s.castRay((5, 5, 15), (0, 0, -1)).tobytes()


@pytest.mark.parametrize("lod", [(0.0, 0.01), (0.0, 0.05), (0.0, 0.2), (0.3, 0.02), (0.0, 1.0)])
def test_lod_is_a_prefix_of_the_full_traversal(vo, lod):
    """castRayWithLOD follows castRay's iterations until the cut fires, so each
    ray either returns the full-detail result unchanged or an LOD hit after no
    more iterations than castRay ran."""
    rng = np.random.default_rng(5)
    R = 64
    bits = (rng.integers(0, 2 ** 63, size=R * R, dtype=np.int64).view(np.uint64) &
            rng.integers(0, 2 ** 63, size=R * R, dtype=np.int64).view(np.uint64))
    s = vo.OracleScene.from_dense(bits, R, 6)
    o = rng.uniform(-32, 96, size=(3000, 3)).astype(np.float32)
    d = rng.normal(size=(3000, 3)).astype(np.float32)
    rays = np.concatenate([o, d], 1)
    full = s.cast_rays(rays)
    cut = s.cast_rays_lod(rays, lod)
    is_lod = ((cut["flags"] & 1) == 1) & (cut["brick"] == 0xFFFFFFFF)
    assert is_lod.any()
    assert cut[~is_lod].tobytes() == full[~is_lod].tobytes()
    assert np.all(cut["iters"][is_lod] <= full["iters"][is_lod])
    assert np.all(cut["flags"][is_lod] == 0x03) and np.all(cut["voxel"][is_lod] == 0xFFFF)
    assert np.all(cut["scale"][is_lod] <= 5)
