"""Host builder (vx_build_dense) against the oracle's restated rebuild (CPU only).

The oracle follows SVORebuild.cpp:228-607 with its hash maps and BFS queue; the
product builder uses the closed form (Morton rank per level).  Both must emit
identical descriptors, brick order, lookup table and occupancy masks.
"""
import numpy as np
import pytest


def _pack(dense):
    R = dense.shape[0]
    flat = dense.reshape(R, R, R // 64, 64)
    w = np.zeros((R, R, R // 64), np.uint64)
    for b in range(64):
        w |= flat[..., b].astype(np.uint64) << np.uint64(b)
    return w.reshape(-1)


FIELDS = ["nodes", "node_brick", "grid_lookup", "brick_coord", "brick_occ"]


@pytest.mark.parametrize("R,levels,p,seed", [(64, 6, 0.001, 1), (64, 7, 0.02, 2), (64, 8, 0.3, 3), (128, 7, 0.0005, 4),
                                              (128, 9, 0.01, 5), (192, 8, 0.002, 6)])
def test_builder_matches_oracle_random(vx, vo, R, levels, p, seed):
    rng = np.random.default_rng(seed)
    dense = rng.random((R, R, R)) < p  # [z, y, x]
    bits = _pack(dense)
    a = vx.build_dense(bits, R, levels)
    e = vo.OracleScene.from_dense(bits, R, levels).export()
    for f in FIELDS:
        np.testing.assert_array_equal(getattr(a, f), e[f], err_msg=f)


@pytest.mark.parametrize("R,levels", [(64, 6), (256, 8)])
def test_builder_matches_oracle_noise(vx, vo, R, levels):
    bits = vx.synth_noise(R, 32 if R >= 128 else 16, 4 if R >= 128 else 3, 0.10, 11, True)
    a = vx.build_dense(bits, R, levels)
    o = vo.OracleScene.from_dense(bits, R, levels)
    e = o.export()
    for f in FIELDS:
        np.testing.assert_array_equal(getattr(a, f), e[f], err_msg=f)
    assert a.node_count == o.node_count and a.brick_count == o.brick_count


def test_dense_and_key_builders_agree(vo):
    # The dense-grid entry point bins exactly like the voxel-list one when
    # world_min = 0 (SVORebuild.cpp:295-302 vs EntityBrickView LocalGrid lookup).
    R = 64
    rng = np.random.default_rng(7)
    dense = rng.random((R, R, R)) < 0.01
    z, y, x = np.nonzero(dense)
    keys = np.stack([x, y, z], 1).astype(np.int32)
    a = vo.OracleScene.from_dense(_pack(dense), R, 6).export()
    b = vo.OracleScene.from_keys(keys, (0, 0, 0), (R, R, R), 6).export()
    for f in FIELDS:
        np.testing.assert_array_equal(a[f], b[f], err_msg=f)


def test_occupancy_mask_layout(vx):
    R = 64
    dense = np.zeros((R, R, R), bool)
    dense[10, 3, 17] = True  # z=10, y=3, x=17 -> brick (2,0,1), local (1,3,2)
    a = vx.build_dense(_pack(dense), R, 6)
    assert a.brick_count == 1
    assert a.brick_coord[0] == 2 | (0 << 10) | (1 << 20)
    i = 2 * 64 + 3 * 8 + 1
    words = a.brick_occ.reshape(-1, 16)[0]
    assert words[i >> 5] == (1 << (i & 31)) and words.sum() == words[i >> 5]
    assert a.grid_lookup[2 + 0 * 8 + 1 * 64] == 0


def test_empty_scene(vx):
    a = vx.build_dense(np.zeros(64 * 64, np.uint64), 64, 6)
    assert a.node_count == 0 and a.brick_count == 0
    assert np.all(a.grid_lookup == 0xFFFFFFFF)


def test_top_level_must_be_single(vx, vo):
    bits = _pack(np.ones((64, 64, 64), bool))
    with pytest.raises(vx.VxError):
        vx.build_dense(bits, 64, 4)  # 8 bricks/axis need 3 levels above the bricks
    with pytest.raises(ValueError):
        vo.OracleScene.from_dense(bits, 64, 4)


def test_nodes_from_reference_layout(vx):
    # ChildDescriptor {childPointer:15, far:1, valid:8, leaf:8 | brick:24, flags:8}
    ref = np.array([(5 | (0xA5 << 16) | (0x0F << 24)) | ((123456 | (7 << 24)) << 32)], np.uint64)
    nodes, nb = vx.nodes_from_reference(ref)
    assert list(nodes) == [5, 0xA5 | (0x0F << 8)]
    assert list(nb) == [123456]
    with pytest.raises(vx.VxError):
        vx.nodes_from_reference(np.array([1 << 15], np.uint64))  # far bit


def test_synth_deterministic(vx):
    a = vx.synth_noise(64, 16, 3, 0.1, 9, True)
    b = vx.synth_noise(64, 16, 3, 0.1, 9, True)
    c = vx.synth_noise(64, 16, 3, 0.1, 10, True)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    n = int(np.unpackbits(vx.synth_noise(64, 16, 3, 0.25, 9, False).view(np.uint8)).sum())
    assert abs(n / 64 ** 3 - 0.25) < 0.001


def test_synth_urban_shape(vx):
    R = 512
    bits = vx.synth_urban(R, 16, 400, 3)
    dense = np.unpackbits(bits.view(np.uint8), bitorder="little").reshape(R, R, R)  # [z, y, x]
    pitch, street = R // 32, max(1, R // 256)
    assert not dense[:, :, pitch - street:pitch].any()          # street in x
    assert not dense[pitch - street:pitch, :, :].any()          # street in z
    col = dense[:pitch - street, :, :pitch - street]
    assert col.any()


def test_tile_order_is_vx_render_lane_order(vx):
    """workloads.tile_order: a permutation of the pixels; 32 x 8 tiles, warps of 8 x 4."""
    from vx_b200 import workloads as W
    for w, h in ((1920, 1080), (100, 37), (33, 9), (8, 4)):
        o = W.tile_order(w, h)
        assert np.array_equal(np.sort(o), np.arange(w * h))
    o = W.tile_order(64, 8)
    first_warp = [y * 64 + x for y in range(4) for x in range(8)]
    assert list(o[:32]) == first_warp
    assert list(o[32:40]) == list(range(8, 16))   # the next warp starts 8 pixels to the right
    assert o[4 * 32] == 4 * 64                    # warp 4 starts 4 rows down
