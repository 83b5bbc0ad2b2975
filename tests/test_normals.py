"""DXT normal payload on the CPU: the oracle's restatement of DXTNormalCompressor
(VoxelData/src/Compression/DXT1Compressor.cpp:168-354) against the reference's
own tests (VoxelData/tests/test_block_compressor.cpp:144-198), geometric normals
(SVO/src/SVORebuild.cpp:145-193), and the product's host builder
(vx_build_normals) bit for bit against the oracle."""
import math

import numpy as np
import pytest


def _unit(v):
    v = np.asarray(v, np.float32)
    return v * (np.float32(1.0) / np.sqrt(np.sum(v * v, axis=-1, keepdims=True, dtype=np.float32)))


def test_up_vector_block(vo):
    """DXTNormalUpVector: 16 x (0,1,0) decode to normals with y > 0.9."""
    a, b = vo.dxtn_encode_block(np.tile(np.float32([0, 1, 0]), (16, 1)))
    out = _unit(vo.dxtn_decode_block(a, b))
    assert np.all(out[:, 1] > 0.9)


def test_varied_block(vo):
    """DXTNormalVaried: a coherent fan keeps at least 8 of 16 within dot > 0.5."""
    inp = []
    for i in range(16):
        ang = np.float32(i) * np.float32(0.4)
        inp.append([math.cos(ang) * 0.3, 0.9, math.sin(ang) * 0.3])
    inp = _unit(np.array(inp, np.float32))
    a, b = vo.dxtn_encode_block(inp)
    out = _unit(vo.dxtn_decode_block(a, b))
    assert np.sum(np.sum(inp * out, 1) > 0.5) >= 8


def test_block_sizes():
    """CalculateCompressedSize: a brick's 512 normals are 32 blocks of 16 bytes."""
    assert 32 * 16 == 512


def test_raw_normal_packing(vo):
    # dominant axis in bits 29-30, its sign in bit 31
    assert vo.encode_raw_normal([0, 1, 0]) >> 29 == 1
    assert vo.encode_raw_normal([0, 0, -1]) >> 29 == 0b110
    assert vo.encode_raw_normal([2, 1, 1]) >> 29 == 0


def test_geometric_normals(vo):
    def i(x, y, z):
        return z * 64 + y * 8 + x

    occ = np.zeros(16, np.uint32)
    for v in (i(3, 3, 3), i(4, 3, 3)):
        occ[v >> 5] |= np.uint32(1 << (v & 31))
    g = vo.geometric_normals(occ)
    np.testing.assert_array_equal(g[i(3, 3, 3)], [-1, 0, 0])  # solid +x neighbour: faces -x
    np.testing.assert_array_equal(g[i(4, 3, 3)], [1, 0, 0])
    np.testing.assert_array_equal(g[i(0, 0, 0)], [0, 1, 0])   # no gradient: (0,1,0)
    full = np.full(16, 0xFFFFFFFF, np.uint32)
    g = vo.geometric_normals(full)
    np.testing.assert_array_equal(g[i(3, 3, 3)], [0, 1, 0])   # interior
    np.testing.assert_allclose(g[i(0, 0, 0)], _unit([-1, -1, -1]), rtol=0, atol=1e-7)  # corner faces out


def _bricks(seed, n):
    rng = np.random.default_rng(seed)
    dens = rng.uniform(0.05, 0.95, size=(n, 1))
    bits = rng.random((n, 512)) < dens
    occ = np.zeros((n, 16), np.uint32)
    for w in range(16):
        occ[:, w] = np.sum(bits[:, 32 * w:32 * w + 32].astype(np.uint64) << np.arange(32, dtype=np.uint64), axis=1)
    occ[0] = 0
    occ[1] = 0xFFFFFFFF
    return occ


def test_host_builder_equals_oracle(vx, vo):
    occ = _bricks(3, 300)
    want = vo.brick_normals(occ)
    got = vx.build_normals(occ)
    np.testing.assert_array_equal(got, want)
    assert np.all(want[0] == 0)  # empty brick: empty blocks


def test_host_builder_noise_scene_equals_oracle(vx, vo):
    from vx_b200 import workloads as W
    wl = W.config1(R=64, width=8, height=8, seed=31)
    occ = wl.scene.brick_occ.reshape(-1, 16)
    np.testing.assert_array_equal(vx.build_normals(occ), vo.brick_normals(occ))


def test_geometric_normals_survive_compression(vo):
    """Decoded normals of occupied surface voxels stay close to their inputs."""
    occ = _bricks(4, 40)
    blocks = vo.brick_normals(occ)
    dots = []
    for b in range(2, 40):
        g = vo.geometric_normals(occ[b])
        for k in range(32):
            dec = _unit(vo.dxtn_decode_block(int(blocks[b, k, 0]), int(blocks[b, k, 1])))
            for t in range(16):
                i = 16 * k + t
                if (occ[b, i >> 5] >> (i & 31)) & 1:
                    dots.append(float(np.dot(dec[t], g[i])))
    assert np.mean(dots) > 0.8


def _colours(seed, n):
    rng = np.random.default_rng(seed)
    rgb = rng.random((n, 512, 3), dtype=np.float32)
    # smooth gradients in half the bricks, as rebuilt scene colours are
    t = np.linspace(0, 1, 512, dtype=np.float32)[None, :, None]
    rgb[::2] = (t * rng.random((n, 1, 3), dtype=np.float32) + (1 - t) * rng.random((n, 1, 3), dtype=np.float32))[::2]
    return rgb


def test_host_dxt1_builder_equals_oracle(vx, vo):
    occ = _bricks(12, 200)
    rgb = _colours(13, 200)
    want = vo.brick_dxt1(rgb, occ)
    np.testing.assert_array_equal(vx.build_dxt1(rgb, occ), want)
    assert np.all(want[:32] == 0)  # empty brick


def test_dxt1_payload_decodes_close(vx, vo):
    """Decoded texels of occupied voxels stay near their colours
    (CompressedBufferRoundTrip, test_block_compressor.cpp:205-240: 0.3)."""
    occ = _bricks(14, 20)
    rgb = _colours(15, 20)
    out = vx.build_dxt1(rgb, occ)
    errs = []
    for b in range(2, 20, 2):
        for k in range(32):
            dec = vo.dxt1_decode_block(int(out[b * 32 + k]))
            for t in range(16):
                i = 16 * k + t
                if (occ[b, i >> 5] >> (i & 31)) & 1:
                    errs.append(float(np.linalg.norm(dec[t] - rgb[b, i])))
    assert np.median(errs) < 0.3


def _shaped_bricks(seed, n):
    """Bricks cut by planes, spheres and thin slabs, plus checkerboards and single
    voxels: many distinct neighbour codes per block and cancelling normals."""
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(np.arange(8), np.arange(8), np.arange(8), indexing="ij")
    p = np.stack([x.ravel(), y.ravel(), z.ravel()], 1).astype(np.float64)
    nrm = rng.normal(size=(n, 3))
    side = p @ nrm.T - rng.uniform(-6, 6, size=n) * np.linalg.norm(nrm, axis=1)
    c = rng.uniform(-2, 10, size=(n, 3))
    sphere = np.linalg.norm(p[:, None] - c[None], axis=2) < rng.uniform(0.5, 8, size=n)
    slab = np.abs(side) < rng.uniform(0.3, 2, size=n)
    cb = ((x + y + z) % 2 == 0).ravel()
    bits = np.concatenate([(side > 0).T, sphere.T, slab.T, np.stack([cb, ~cb, np.eye(512, dtype=bool)[5],
                                                                     np.eye(512, dtype=bool)[511]])])
    occ = np.zeros((bits.shape[0], 16), np.uint32)
    for w in range(16):
        occ[:, w] = np.sum(bits[:, 32 * w:32 * w + 32].astype(np.uint64) << np.arange(32, dtype=np.uint64), axis=1)
    return occ


def test_host_builder_shaped_bricks_equal_oracle(vx, vo):
    """The host builder looks normals up by neighbour code and searches distinct
    codes only; the oracle evaluates every texel."""
    occ = _shaped_bricks(5, 1500)
    np.testing.assert_array_equal(vx.build_normals(occ), vo.brick_normals(occ))
