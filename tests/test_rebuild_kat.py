"""RebuildHierarchyTest (SVO/tests/test_rebuild_hierarchy.cpp) on the oracle's restated
rebuild, with the device-format export the product uses: brick views, descriptor counts, root
masks and child pointers; the 64^3 noise case also through the product's own builder."""
import numpy as np


def _root(o):
    e = o.export()
    return int(e["nodes"][0]), int(e["nodes"][1]) & 0xFF, (int(e["nodes"][1]) >> 8) & 0xFF


def test_multiple_bricks_hierarchy(vo):
    """:26-106 - 8 voxels in 4 bricks of a 32^3 world, depth 8."""
    pts = [(2, 2, 2), (5, 5, 5), (18, 2, 2), (20, 5, 5), (2, 18, 2), (5, 20, 5), (18, 18, 2), (20, 20, 5)]
    o = vo.OracleScene.from_positions(pts, (0, 0, 0), (32, 32, 32), 8)
    assert o.brick_count >= 4
    assert o.node_count > o.brick_count
    child, valid, leaf = _root(o)
    assert valid > 0 and leaf == 0x00
    if child > 0:
        assert child < o.node_count


def test_single_brick(vo):
    """:110-148 - two voxels in one brick of a 16^3 world."""
    o = vo.OracleScene.from_positions([(2, 2, 2), (3, 3, 3)], (0, 0, 0), (16, 16, 16), 8)
    assert o.brick_count == 1
    assert o.node_count >= 1


def test_empty_world(vo):
    """:152-176 - no voxels: no brick views, no descriptors."""
    o = vo.OracleScene.from_keys(np.zeros((0, 3), np.int32), (0, 0, 0), (16, 16, 16), 8)
    assert o.brick_count == 0 and o.node_count == 0


def _noise_terrain():
    """noise3D of :192-197 in int32 arithmetic (C++ wraps on these targets) and the sampling
    loop of :206-224 (every second voxel, vertical falloff, threshold 0.3)."""
    pts = []
    for z in range(0, 64, 2):
        for y in range(0, 64, 2):
            for x in range(0, 64, 2):
                n = np.int32(x + y * 57 + z * 997)
                with np.errstate(over="ignore"):
                    n = np.int32((n << np.int32(13)) ^ n)
                    m = np.int32(n * np.int32(n * n * np.int32(15731) + np.int32(789221)) + np.int32(1376312589))
                v = np.float32(1.0) - np.float32(int(m) & 0x7FFFFFFF) / np.float32(1073741824.0)
                h = np.float32(1.0) - np.float32(y) / np.float32(64)
                if v * np.float32(0.5) + h * np.float32(0.5) > np.float32(0.3):
                    pts.append((x, y, z))
    return pts


def test_stress_noise_generated(vx, vo):
    """:180-262 - sparse 64^3 terrain: bricks, descriptors, a root with valid children; the
    product's builder gives the same arrays from the same voxels."""
    pts = _noise_terrain()
    assert len(pts) > 0
    o = vo.OracleScene.from_positions(pts, (0, 0, 0), (64, 64, 64), 8)
    assert o.brick_count > 0 and o.node_count > 0
    assert _root(o)[1] > 0
    R = 64
    bits = np.zeros(R * R * (R // 64), np.uint64)
    for x, y, z in pts:
        bits[(z * R + y) * (R // 64) + x // 64] |= np.uint64(1) << np.uint64(x % 64)
    a = vx.build_dense(bits, R, 8)
    e = o.export()
    for k in ("nodes", "node_brick", "grid_lookup", "brick_coord", "brick_occ"):
        np.testing.assert_array_equal(getattr(a, k), e[k], err_msg=k)
