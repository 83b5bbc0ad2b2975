"""Material-ID colour on the GPU (needs a B200): a scene whose colour is the reference's
per-voxel material words (VX_COLOR_MATERIAL) renders pixels equal to the oracle's shading of
getMaterialColor(word & 0xFF) (shaders/Materials.glsl:18-60, VoxelRayMarch.comp:188-192) bit
for bit, the cast reports each hit's word, a scene loaded from a VSCA file renders the same,
and the device DXT1 payload built from the words (MaterialIdToColor) equals the oracle's."""
import numpy as np
import pytest

from test_cache import _pack_vsca
from test_gpu_parity import assert_hits_equal
from test_materials import material_words

pytestmark = pytest.mark.gpu


def _render_and_check(vx, vo, arrays, bits, R, words, cam, w, h):
    import torch
    s = vx.Scene(arrays)
    n = w * h
    img = torch.zeros(n, dtype=torch.int32, device="cuda")
    hits = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    col = torch.zeros((n, 1), dtype=torch.int32, device="cuda")
    s.render_dev(cam, w, h, img, hits, col)
    torch.cuda.synchronize()
    o = vo.OracleScene.from_dense(bits, R, arrays.max_levels)
    rays, uv_y = vo.camera_rays(cam, w, h, with_uv_y=True)
    oh = o.cast_rays(rays)
    assert_hits_equal(hits.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1), oh, None, "material render hits")
    hit = (oh["flags"] & 1).astype(bool)
    assert hit.mean() > 0.05
    want_word = np.zeros(n, np.uint32)
    want_word[hit] = words[oh["brick"][hit].astype(np.int64) * 512 + oh["voxel"][hit]]
    np.testing.assert_array_equal(col.cpu().numpy()[:, 0].view(np.uint32), want_word)
    image = img.cpu().numpy().view(np.uint32)
    palette = {}
    for i in range(n):
        if hit[i]:
            m = int(want_word[i]) & 0xFF
            if m not in palette:
                palette[m] = vo.material_color(m, shader=True)
            c = palette[m]
        else:
            c = np.zeros(3, np.float32)
        want = vo.shade(c, bool(hit[i]), (int(oh["flags"][i]) >> 1) & 3, bool(oh["flags"][i] & 8), float(uv_y[i]))
        assert image[i] == want, (i, hex(image[i]), hex(want))
    return len(palette)


def test_material_scene_renders_like_the_shader(vx, vo, cuda):
    from vx_b200 import workloads as W
    R = 128
    bits = vx.synth_noise(R, 16, 3, 0.4, 12, False)
    a = W.scene_from_bits(bits, R, None, 12)
    words = material_words(a.brick_occ, 6)
    a.color_kind, a.brick_color = vx.VX_COLOR_MATERIAL, words
    cam = W.empty_voxel_camera(bits, R, 12, 70.0, 96, 72)
    assert _render_and_check(vx, vo, a, bits, R, words, cam, 96, 72) >= 5  # several palette entries reached


def test_vsca_loaded_material_scene_renders_like_the_shader(vx, vo, cuda, tmp_path):
    from vx_b200 import workloads as W
    R = 64
    bits = vx.synth_noise(R, 8, 3, 0.35, 14, False)
    a = W.scene_from_bits(bits, R, None, 14)
    words = material_words(a.brick_occ, 7)
    p = tmp_path / "m.vsca"
    p.write_bytes(_pack_vsca([{"arrays": a, "ci": (1, R, 0.35, 14), "words": words}]))
    b = vx.cache_read_vsca(str(p))
    assert b.color_kind == vx.VX_COLOR_MATERIAL
    cam = W.empty_voxel_camera(bits, R, 14, 70.0, 80, 60)
    _render_and_check(vx, vo, b, bits, R, words, cam, 80, 60)


def test_device_dxt1_payload_from_materials_equals_oracle(vx, vo, cuda):
    import torch
    from vx_b200 import workloads as W
    bits = vx.synth_noise(128, 16, 3, 0.5, 15, False)
    a = W.scene_from_bits(bits, 128, None, 15)
    words = material_words(a.brick_occ, 8)
    B = a.brick_count
    d_words = torch.from_numpy(words.view(np.int32)).cuda()
    d_rgb = torch.zeros(B * 512 * 3, dtype=torch.float32, device="cuda")
    vx.material_rgb_dev(d_words, d_rgb)
    d_occ = torch.from_numpy(a.brick_occ.view(np.int32)).cuda()
    d_out = torch.zeros(B * 32, dtype=torch.int64, device="cuda")
    vx.build_dxt1_dev(d_rgb, d_occ, d_out)
    torch.cuda.synchronize()
    rgb = d_rgb.cpu().numpy()
    np.testing.assert_array_equal(rgb.view(np.uint32), vx.material_rgb(words).reshape(-1).view(np.uint32))
    np.testing.assert_array_equal(d_out.cpu().numpy().view(np.uint64), vo.brick_dxt1(rgb, a.brick_occ))
