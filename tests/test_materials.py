"""Material-ID colour, the reference's own colour source (CPU).

The reference stores a material word per voxel (brickData,
CashSystem/src/VoxelSceneCacher.cpp:500, 586-587).  Its uncompressed shader colours a hit
with getMaterialColor(word & 0xFF) (shaders/Materials.glsl:18-60) and its compressed payload
is encoded from MaterialIdToColor(id) (SVO/src/SVORebuild.cpp:68-120, 679-700); the two
tables differ on ids 33-39.  Checked here: the library's payload colours equal the oracle's
MaterialIdToColor, the DXT1 payload built from them equals the oracle's encoder, and VSCA
files keep the words (read from the reference's layout and written back)."""
import numpy as np
import pytest

from test_cache import _pack_vsca, _same

IDS = np.array(list(range(0, 70)) + [99, 100, 127, 128, 200, 255, 256, 257, 1000, 0xFFFFFFFF], np.uint32)


def material_words(brick_occ, seed):
    """Seeded material ids for the occupied voxels of bricks (0 for empty voxels); ids cover
    every palette branch: the listed Cornell, stone and city ids and the colour wheel."""
    rng = np.random.default_rng(seed)
    pool = np.array([1, 2, 3, 4, 5, 6, 7, 10, 11, 20] + list(range(30, 41)) + [50, 60, 61] + list(range(100, 256, 7)),
                    np.uint32)
    B = brick_occ.size // 16
    occ = np.unpackbits(np.ascontiguousarray(brick_occ, np.uint32).reshape(B, 16).view(np.uint8), axis=1,
                        bitorder="little").reshape(-1)
    return np.where(occ == 1, rng.choice(pool, size=occ.size), 0).astype(np.uint32)


def test_payload_colours_equal_oracle(vx, vo):
    got = vx.material_rgb(IDS)
    for k, i in enumerate(IDS):
        np.testing.assert_array_equal(got[k].view(np.uint32), vo.material_color(int(i)).view(np.uint32), err_msg=int(i))
    # the two tables agree except on the interpolated stone ids 33-39 (37 happens to agree)
    differ = [int(i) for i in range(256) if not np.array_equal(vo.material_color(i), vo.material_color(i, True))]
    assert set(differ) <= set(range(33, 40)) and len(differ) >= 5


def test_dxt1_payload_from_materials_equals_oracle(vx, vo):
    from vx_b200 import workloads as W
    bits = vx.synth_noise(64, 8, 3, 0.4, 5, False)
    a = W.scene_from_bits(bits, 64, None, 5)
    words = material_words(a.brick_occ, 3)
    rgb = vx.material_rgb(words)
    want_rgb = np.stack([vo.material_color(int(w)) for w in words[:4096]])
    np.testing.assert_array_equal(rgb[:4096].view(np.uint32), want_rgb.view(np.uint32))
    got = vx.build_dxt1(rgb.reshape(-1, 512, 3), a.brick_occ)
    np.testing.assert_array_equal(got, vo.brick_dxt1(rgb.reshape(-1), a.brick_occ))


def test_vsca_keeps_material_words(vx, tmp_path):
    """A file packed in the reference's layout with per-voxel material ids and no colour
    section reads back with the words as its colour (VX_COLOR_MATERIAL) and occupancy
    word != 0; a file with DXT1 colours gives them by default and the words on request; the
    writer stores a material scene's words as brickData, byte for byte the reference's layout."""
    from vx_b200 import workloads as W
    bits = vx.synth_noise(64, 8, 3, 0.3, 8, False)
    a = W.scene_from_bits(bits, 64, "dxt1", 8)
    words = material_words(a.brick_occ, 4)
    p = tmp_path / "m.vsca"
    plain = W.scene_from_bits(bits, 64, None, 8)
    p.write_bytes(_pack_vsca([{"arrays": plain, "ci": (1, 64, 0.3, 8), "words": words}]))
    b = vx.cache_read_vsca(str(p))
    assert b.color_kind == vx.VX_COLOR_MATERIAL
    np.testing.assert_array_equal(b.brick_color, words)
    _same(plain, b, color=False, normals=False)
    q = tmp_path / "md.vsca"
    q.write_bytes(_pack_vsca([{"arrays": a, "ci": (1, 64, 0.3, 8), "words": words}]))
    c = vx.cache_read_vsca(str(q))
    assert c.color_kind == vx.VX_COLOR_DXT1
    np.testing.assert_array_equal(c.brick_color, a.brick_color)
    m = vx.cache_read_vsca(str(q), materials=True)
    assert m.color_kind == vx.VX_COLOR_MATERIAL
    np.testing.assert_array_equal(m.brick_color, words)
    # writer: a VX_COLOR_MATERIAL scene's words become brickData
    plain.color_kind, plain.brick_color = vx.VX_COLOR_MATERIAL, words
    r = tmp_path / "w.vsca"
    vx.cache_write_vsca(str(r), plain, 1, 64, 0.3, 8)
    plain.brick_color = None
    plain.color_kind = vx.VX_COLOR_NONE
    assert r.read_bytes() == _pack_vsca([{"arrays": plain, "ci": (1, 64, 0.3, 8), "words": words, "n_materials": 0}])
    # an occupied voxel with word 0 cannot be written (the reference reads word 0 as empty)
    bad = words.copy()
    bad[np.flatnonzero(bad)[0]] = 0
    plain.color_kind, plain.brick_color = vx.VX_COLOR_MATERIAL, bad
    with pytest.raises(vx.VxError):
        vx.cache_write_vsca(str(tmp_path / "bad.vsca"), plain, 1, 64, 0.3, 8)
