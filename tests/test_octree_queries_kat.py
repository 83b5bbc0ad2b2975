"""The castRay cases of OctreeQueryTest (SVO/tests/test_octree_queries.cpp:175-400) on its
hand-built octree (:23-78: a root whose only child, octant 0, has 8 leaf children; world
[0,10]^3, maxLevels 4, no brick data).  CPU: the oracle meets every assertion.  GPU: the kernel
returns the oracle's records for the same rays."""
import numpy as np
import pytest

FLT_MAX = 3.4028234663852886e38


def _fixture_nodes():
    # {child_ptr, valid | leaf << 8} for root (childPointer 1, valid 0b1) and the leaf parent
    return np.array([1, 0x01, 0, 0xFF | (0xFF << 8)], np.uint32)


def _norm(v):
    v = np.asarray(v, np.float32)
    return v * (np.float32(1.0) / np.sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]))


# (name, origin, direction, tMin, tMax, reference line)
MISSES = [
    ("CastRayMissEmpty", (7, 7, 7), (1, 0, 0), 0.0, 10.0, 175),
    ("CastRayMissOutsideBounds", (-5, 15, 5), (1, 0, 0), 0.0, 10.0, 185),
    ("CastRayZeroDirection", (1, 1, 1), (0, 0, 0), 0.0, FLT_MAX, 198),
    ("CompleteMiss_Above", (-5, 15, 5), (1, 0, 0), 0.0, FLT_MAX, 282),
    ("CompleteMiss_Below", (-5, -5, 5), (1, 0, 0), 0.0, FLT_MAX, 291),
    ("CompleteMiss_Left", (-5, 5, -5), (0, 0, 1), 0.0, FLT_MAX, 300),
    ("CompleteMiss_DiagonalPast", (-5, -5, -5), tuple(_norm((1, -0.5, -0.5))), 0.0, FLT_MAX, 308),
    ("Miss_OppositeDirection", (-5, 5, 5), (-1, 0, 0), 0.0, FLT_MAX, 317),
    ("EntryExit_ThroughEmptyRegion", (-5, 7, 7), (1, 0, 0), 0.0, FLT_MAX, 330),
    ("Range_StartBeyondGrid", (-5, 2.5, 2.5), (1, 0, 0), 20.0, FLT_MAX, 343),
    ("Range_EndBeforeGrid", (-5, 2.5, 2.5), (1, 0, 0), 0.0, 3.0, 353),
    ("Numerical_VeryShortRay", (-1, 2.5, 2.5), (1, 0, 0), 0.0, 0.1, 373),
]


def _scene(vo):
    return vo.OracleScene.from_descriptors(_fixture_nodes(), None, (0, 0, 0), (10, 10, 10), 4)


@pytest.mark.parametrize("case", MISSES, ids=[m[0] for m in MISSES])
def test_fixture_misses(vo, case):
    name, o, d, tmin, tmax, _ = case
    h = _scene(vo).castRay(o, d, tmin, tmax)
    assert not (h["flags"] & 1), name


def test_fixture_near_miss_and_lod_zero_bias(vo):
    s = _scene(vo)
    h = s.castRay((-1, 5.01, 2.5), (1, 0, 0))                    # Complex_NearMiss (:381-400)
    assert (not (h["flags"] & 1)) or h["t"] > 0.0
    a = s.castRayLOD((-1, 1, 1), (1, 0, 0), 0.0)                 # CastRayLODZeroBias (:209-220)
    b = s.castRay((-1, 1, 1), (1, 0, 0))
    assert bool(a["flags"] & 1) == bool(b["flags"] & 1)
    if a["flags"] & 1:
        assert abs(float(a["t"]) - float(b["t"])) < 0.01 and a["scale"] == b["scale"]


@pytest.mark.gpu
def test_fixture_kernel_equals_oracle(vx, vo, cuda):
    from test_gpu_parity import assert_hits_equal, gpu_cast, scene_from_oracle
    from vx_b200 import workloads as W
    o = _scene(vo)
    a = scene_from_oracle(vx, o, ((0, 0, 0), (10, 10, 10)), 4)
    rays = np.array([list(m[1]) + list(m[2]) for m in MISSES] + [[-1, 5.01, 2.5, 1, 0, 0], [-1, 1, 1, 1, 0, 0]],
                    np.float32)
    rays = np.concatenate([rays, W.random_rays(3000, 10.0, seed=31, lo=-0.5, hi=1.5)])
    for tmin, tmax in ((0.0, FLT_MAX), (0.0, 10.0), (20.0, FLT_MAX), (0.0, 3.0)):
        g, _, cnt = gpu_cast(vx, a, rays, tmin, tmax)
        assert_hits_equal(g, o.cast_rays(rays, tmin, tmax), cnt, f"fixture t in [{tmin},{tmax}]")
