"""Known-answer cases ported from the reference's ray-casting tests.

Each case restates one assertion block of
  VIXEN/libraries/SVO/tests/test_ray_casting_comprehensive.cpp
  VIXEN/libraries/SVO/tests/test_brick_traversal.cpp
with the same voxel set, world bounds, octree depth and ray.  `expect` is the
reference test's assertion on the returned RayHit.  `diverges` names cases
where the restated reference code does not meet the reference test's own
assertion (the reference cannot be built here, so its tests cannot be re-run);
for those the oracle's outcome is pinned instead, with the reason.
"""
import numpy as np


def _norm(v):
    v = np.asarray(v, np.float32)
    return tuple(v * (np.float32(1.0) / np.sqrt(np.float32((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]))))


def near(p, q, tol):
    return float(np.linalg.norm(np.asarray(p, np.float64) - np.asarray(q, np.float64))) < tol


class Case:
    def __init__(self, name, voxels, depth, origin, direction, expect, tmin=0.0, tmax=100.0, bounds=None,
                 diverges=None):
        self.name = name
        self.voxels = [tuple(float(c) for c in v) for v in voxels]
        self.depth = depth
        self.origin = tuple(float(c) for c in origin)
        self.direction = tuple(float(c) for c in direction)
        self.expect = expect
        self.tmin, self.tmax = tmin, tmax
        v = np.asarray(self.voxels, np.float32)
        if bounds is None:  # createOctreeWithVoxels: voxel AABB padded by 1 (test_ray_casting_comprehensive.cpp:37-55)
            self.world_min = tuple(v.min(0) - 1)
            self.world_max = tuple(v.max(0) + 1)
        else:
            self.world_min, self.world_max = bounds
        self.diverges = diverges


def hit(h):
    return bool(h["flags"] & 1)


def _hollow_cube():
    vox = []
    for y in range(1, 10):
        for z in range(1, 10):
            vox += [(1, y, z), (9, y, z)]
    for x in range(2, 9):
        for z in range(1, 10):
            vox += [(x, 1, z), (x, 9, z)]
    for x in range(2, 9):
        for y in range(2, 9):
            vox += [(x, y, 1), (x, y, 9)]
    return vox


def _dense(lo, hi):
    return [(x, y, z) for x in range(lo, hi + 1) for y in range(lo, hi + 1) for z in range(lo, hi + 1)]


def _cornell_small():
    walls = [(x, y, 7) for x in range(1, 7) for y in range(1, 7)]
    walls += [(1, y, z) for y in range(1, 7) for z in range(1, 7)]
    walls += [(6, y, z) for y in range(1, 7) for z in range(1, 7)]
    walls += [(x, 1, z) for x in range(2, 6) for z in range(1, 7)]
    walls += [(x, 6, z) for x in range(2, 6) for z in range(1, 7)]
    objs = [(x, y, z) for x in range(3, 5) for y in range(2, 4) for z in range(3, 5)]
    return walls + objs


W10 = ((0.0, 0.0, 0.0), (10.0, 10.0, 10.0))  # BrickTraversalTest bounds (test_brick_traversal.cpp:24-25)
HOLLOW_DIVERGES = ("world 10^3 gives 2 bricks per axis but 5-voxel ESVO cells: the position-based brick lookup "
                   "(SVOBrickDDA.cpp:126-136) maps the far cell to brick 0 again, so the right wall in brick 1 is "
                   "never marched")
BOUNDARY_DIVERGES = ("world 10^3 gives 2 bricks per axis but 5-voxel ESVO cells: a ray on y = z = 5 starts in the "
                     "upper y/z octants (selectInitialOctant, SVOTraversal.cpp:747-763), whose valid bits are clear "
                     "because the only brick, grid (0,0,0), is the root's octant 0")

CASES = [
    # --- TEST 1 AxisAlignedRaysFromOutside (:105-174)
    *[Case(f"axis_{i}", [(5, 2, 2), (2, 5, 2), (2, 2, 5), (8, 8, 8)], 6, o, d,
           (lambda tgt: (lambda h: hit(h) and near(h["hit_point"], tgt, 5.0)))(t))
      for i, (o, d, t) in enumerate([((-5, 2, 2), (1, 0, 0), (5, 2, 2)), ((15, 8, 8), (-1, 0, 0), (8, 8, 8)),
                                     ((2, -5, 2), (0, 1, 0), (2, 5, 2)), ((8, 15, 8), (0, -1, 0), (8, 8, 8)),
                                     ((2, 2, -5), (0, 0, 1), (2, 2, 5)), ((8, 8, 15), (0, 0, -1), (8, 8, 8))])],
    # --- TEST 2 DiagonalRaysVariousAngles (:179-233)
    Case("diag_111", [(2, 2, 2), (5, 5, 5), (8, 8, 8), (3, 7, 4)], 6, (-2, -2, -2), _norm((1, 1, 1)),
         lambda h: hit(h) and any(near(h["hit_point"], t, 5.0) for t in [(2, 2, 2), (5, 5, 5), (8, 8, 8)])),
    *[Case(f"diag_cond_{i}", [(2, 2, 2), (5, 5, 5), (8, 8, 8), (3, 7, 4)], 6, o, _norm(d),
           lambda h: (not hit(h)) or any(near(h["hit_point"], t, 5.0)
                                         for t in [(2, 2, 2), (5, 5, 5), (8, 8, 8), (3, 7, 4)]))
      for i, (o, d) in enumerate([((-2, 3, 5), (2, 0.5, 0)), ((5, -2, -2), (0, 1, 2)),
                                  ((-1, -1, -1), (2.5, 3.7, 2.1))])],
    # --- TEST 3 RaysFromInsideGrid (:238-304)
    Case("inside_px", _hollow_cube(), 6, (5, 5, 5), (1, 0, 0),
         lambda h: hit(h) and abs(h["hit_point"][0] - 9.0) <= 2.0, diverges=HOLLOW_DIVERGES),
    Case("inside_ny", _hollow_cube(), 6, (5, 5, 5), (0, -1, 0),
         lambda h: hit(h) and abs(h["hit_point"][1] - 1.0) <= 2.0),
    Case("inside_diag", _hollow_cube(), 6, (5, 5, 5), _norm((1, 1, 1)),
         lambda h: hit(h) and all(h["hit_point"][k] > 7.0 for k in range(3)), diverges=HOLLOW_DIVERGES),
    Case("inside_between", _hollow_cube(), 6, (2, 5, 5), (1, 0, 0),
         lambda h: hit(h) and abs(h["hit_point"][0] - 9.0) <= 2.0, diverges=HOLLOW_DIVERGES),
    # --- TEST 4 CompleteMissCases (:309-364)
    Case("miss_above", [(5, 5, 5), (2, 2, 2), (8, 8, 8)], 6, (-5, 15, 5), (1, 0, 0), lambda h: not hit(h)),
    Case("miss_below", [(5, 5, 5), (2, 2, 2), (8, 8, 8)], 6, (5, -5, 5), (0, 0, 1), lambda h: not hit(h)),
    Case("miss_away", [(5, 5, 5), (2, 2, 2), (8, 8, 8)], 6, (15, 15, 15), (1, 1, 1), lambda h: not hit(h)),
    Case("miss_sparse", [(5, 5, 5), (2, 2, 2), (8, 8, 8)], 6, (-1, 3.7, 3.7), (1, 0, 0),
         lambda h: (not hit(h)) or any(near(h["hit_point"], t, 5.0) for t in [(5, 5, 5), (2, 2, 2), (8, 8, 8)])),
    Case("miss_range", [(5, 5, 5), (2, 2, 2), (8, 8, 8)], 6, (-5, 5, 5), (1, 0, 0), lambda h: not hit(h),
         tmax=2.0),
    # --- TEST 5 MultipleVoxelTraversal (:369-405)
    Case("line_first", [(x, 5, 5) for x in range(1, 10)], 6, (-2, 5, 5), (1, 0, 0),
         lambda h: hit(h) and h["hit_point"][0] < 3.0, diverges=BOUNDARY_DIVERGES),
    Case("grid_diag", [(x, y, 5) for x in range(2, 9, 2) for y in range(2, 9, 2)], 6, (0, 0, 5), _norm((1, 1, 0)),
         lambda h: hit(h) and any(near(h["hit_point"], (x, y, 5), 3.0) for x in range(2, 9, 2)
                                  for y in range(2, 9, 2))),
    # --- TEST 6 DenseVolumeTraversal (:410-454)
    Case("dense_front", _dense(3, 7), 8, (5, 5, 0), (0, 0, 1), lambda h: hit(h) and abs(h["hit_point"][2] - 3) <= 2),
    Case("dense_corner", _dense(3, 7), 8, (0, 0, 0), _norm((1, 1, 1)),
         lambda h: hit(h) and all(abs(h["hit_point"][k] - 3) <= 2 for k in range(3))),
    Case("dense_graze", _dense(3, 7), 8, (2.9, 5, 0), (0, 0, 1),
         lambda h: (not hit(h)) or any(near(h["hit_point"], v, 3.0) for v in _dense(3, 7))),
    # --- TEST 7 EdgeCasesAndBoundaries (:459-509)
    Case("edge_center", [(1, 1, 1), (9, 9, 9), (5, 5, 5)], 6, (-2, 5, 5), (1, 0, 0),
         lambda h: hit(h) and near(h["hit_point"], (5, 5, 5), 5.0)),
    Case("edge_corner", [(1, 1, 1), (9, 9, 9), (5, 5, 5)], 6, (0, 0, 0), _norm((1, 1, 1)),
         lambda h: hit(h) and any(near(h["hit_point"], v, 5.0) for v in [(1, 1, 1), (9, 9, 9), (5, 5, 5)])),
    Case("edge_zero_dir", [(1, 1, 1), (9, 9, 9), (5, 5, 5)], 6, (5, 5, 5), (0, 0, 0), lambda h: not hit(h)),
    Case("edge_small", [(1, 1, 1), (9, 9, 9), (5, 5, 5)], 6, (-1, 5, 5), _norm((1, 0.0001, 0.0001)),
         lambda h: (not hit(h)) or any(near(h["hit_point"], v, 5.0) for v in [(1, 1, 1), (9, 9, 9), (5, 5, 5)])),
    # --- TEST 9 PerformanceCharacteristics (:564-587): depth 4..10
    *[Case(f"depth_{dpt}", [(5, 5, 5), (2.5, 2.5, 2.5), (7.5, 7.5, 7.5)], dpt, (0, 0, 0), _norm((1, 1, 1)),
           (lambda dd: (lambda h: hit(h) and (dd < 8 or h["scale"] <= 23 - dd + 2)))(dpt))
      for dpt in (4, 6, 8, 10)],
    # --- TEST 10 CornellBoxScene (:592-691)
    Case("cornell_front", _cornell_small(), 8, (4, 4, -2), (0, 0, 1), lambda h: hit(h) and h["hit_point"][2] > 2.0),
    Case("cornell_above", _cornell_small(), 8, (4, 5, -2), (0, 0, 1),
         lambda h: hit(h) and abs(h["hit_point"][2] - 7.0) <= 2.0),
    Case("cornell_shadow", _cornell_small(), 8, (4, 4, 4), (0, 1, 0),
         lambda h: hit(h) and abs(h["hit_point"][1] - 6.0) <= 2.0),
    Case("cornell_bounce", _cornell_small(), 8, (2, 4, 4), _norm((1, 0.2, 0.3)), lambda h: hit(h)),
    # --- test_brick_traversal.cpp (world [0,10]^3, depth 8)
    Case("brick_leaf", [(5, 5, 5), (5.1, 5.1, 5.1), (5.2, 5.2, 5.2)], 8, (-2, 5, 5), (1, 0, 0),
         lambda h: hit(h) and all(abs(h["hit_point"][k] - 5) <= 2 for k in range(3)), bounds=W10,
         diverges=BOUNDARY_DIVERGES),
    Case("brick_miss_return", [(2, 2, 2), (8, 8, 8)], 8, (-2, 8, 8), (1, 0, 0),
         lambda h: hit(h) and all(abs(h["hit_point"][k] - 8) <= 2 for k in range(3)), bounds=W10),
    Case("brick_multi", [(x, 5, 5) for x in range(1, 10)], 8, (-2, 5, 5), (1, 0, 0),
         lambda h: hit(h) and h["hit_point"][0] < 3.0 and abs(h["hit_point"][1] - 5) <= 1, bounds=W10,
         diverges=BOUNDARY_DIVERGES),
    Case("brick_graze", [(2.5, 2.5, 2.5)], 8, (2.49, 2.0, 0.0), _norm((0.01, 0.5, 1.0)),
         lambda h: (not hit(h)) or abs(h["hit_point"][0] - 2.5) <= 2.0, bounds=W10),
    Case("brick_to_brick", [(2, 5, 5), (7, 5, 5)], 8, (-2, 5, 5), (1, 0, 0),
         lambda h: hit(h) and abs(h["hit_point"][0] - 2) <= 2, bounds=W10, diverges=BOUNDARY_DIVERGES),
]


def axis_parallel_voxels():
    vals = np.arange(2.0, 4.01, 0.5)
    return [(x, y, z) for x in vals for y in vals for z in vals]


CASES += [
    Case(f"brick_axis_{i}", axis_parallel_voxels(), 8, o, d, f, bounds=W10)
    for i, (o, d, f) in enumerate([
        ((0, 3, 3), (1, 0, 0), lambda h: hit(h) and abs(h["hit_point"][1] - 3) <= 1 and abs(h["hit_point"][2] - 3) <= 1),
        ((3, 0, 3), (0, 1, 0), lambda h: hit(h) and abs(h["hit_point"][0] - 3) <= 1 and abs(h["hit_point"][2] - 3) <= 1),
        ((3, 3, 0), (0, 0, 1), lambda h: hit(h) and abs(h["hit_point"][0] - 3) <= 1 and abs(h["hit_point"][1] - 3) <= 1),
    ])
]


def cornell_box_voxels():
    """CornellBoxTest::buildCornellBox (test_cornell_box.cpp:66-136): float positions with
    step 0.5 and wall thickness 0.2 in a 10^3 box (the loops' float32 accumulation is exact), in
    creation order, each with its wall colour."""
    f = np.float32
    size, thick, step = f(10.0), f(0.2), f(0.5)
    grey, red, green, white = (0.8, 0.8, 0.8), (0.8, 0.1, 0.1), (0.1, 0.8, 0.1), (1.0, 1.0, 1.0)

    def rng(lo, hi):
        out, v = [], f(lo)
        while v < hi:
            out.append(float(v))
            v = f(v + step)
        return out
    vox = []
    for x in rng(0, size):
        for z in rng(0, size):
            for y in rng(0, thick):
                vox.append(((x, y, z), grey))
    for x in rng(0, size):
        for z in rng(0, size):
            for y in rng(size - thick, size):
                d = np.hypot(f(x) - f(5.0), f(z) - f(5.0))
                vox.append(((x, y, z), white if d < 2.0 else grey))
    for y in rng(0, size):
        for z in rng(0, size):
            for x in rng(0, thick):
                vox.append(((x, y, z), red))
    for y in rng(0, size):
        for z in rng(0, size):
            for x in rng(size - thick, size):
                vox.append(((x, y, z), green))
    for x in rng(0, size):
        for y in rng(0, size):
            for z in rng(size - thick, size):
                vox.append(((x, y, z), grey))
    return vox


_CB = [p for p, _ in cornell_box_voxels()]
FACE_DIVERGES = ("positions quantise to integer keys (floor(p + 1e-5), MortonCode64::fromWorldPos), so the floor and "
                 "left-wall voxels span [0, 1) and the traversal reports the entry face at exactly 1.0; the test's "
                 "strict < 1.0 fails on the restated code (traverseBrickView, SVOBrickDDA.cpp:492-507)")
CB_BOUNDS = ((0.0, 0.0, 0.0), (10.0, 10.0, 10.0))  # rebuild(world, vec3(0), vec3(boxSize)) (:52)

# --- test_cornell_box.cpp (depth 8): every assertion there is conditional on a hit
CASES += [
    Case("cbox_floor", _CB, 8, (5, 5, 5), (0, -1, 0), lambda h: (not hit(h)) or h["hit_point"][1] < 1.0,
         bounds=CB_BOUNDS, diverges=FACE_DIVERGES),                                                                # :152-164, :290-322
    Case("cbox_ceiling", _CB, 8, (5, 5, 5), (0, 1, 0), lambda h: (not hit(h)) or h["hit_point"][1] > 9.0,
         bounds=CB_BOUNDS),                                                                # :169-181
    Case("cbox_left", _CB, 8, (5, 5, 5), (-1, 0, 0), lambda h: (not hit(h)) or h["hit_point"][0] < 1.0,
         bounds=CB_BOUNDS, diverges=FACE_DIVERGES),                                                                # :186-207
    Case("cbox_right", _CB, 8, (5, 5, 5), (1, 0, 0), lambda h: (not hit(h)) or h["hit_point"][0] > 9.0,
         bounds=CB_BOUNDS),                                                                # :212-233
    Case("cbox_back", _CB, 8, (5, 5, 5), (0, 0, 1), lambda h: (not hit(h)) or h["hit_point"][2] > 9.0,
         bounds=CB_BOUNDS),                                                                # :238-250
    Case("cbox_diagonal", _CB, 8, (1, 1, 1), _norm((1, 1, 1)), lambda h: True, bounds=CB_BOUNDS),  # :255-267
    Case("cbox_outside", _CB, 8, (-5, 5, 5), (-1, 0, 0), lambda h: True, bounds=CB_BOUNDS),       # :272-285
]
