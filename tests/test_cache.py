"""Scene cache files on the CPU: the library's VXSC format round-trips every
array exactly and rejects damaged files; the reference's VSCA format
(VoxelSceneCacher::SerializeToFile / DeserializeFromFile,
CashSystem/src/VoxelSceneCacher.cpp:179-364) is read from files packed here
field by field in the reference's order, and written files read back."""
import struct

import numpy as np
import pytest

FIELDS = ["nodes", "node_brick", "grid_lookup", "brick_coord", "brick_occ"]


def _scene(vx, color="dxt1", R=64, seed=3, normals=True):
    from vx_b200 import workloads as W
    bits = vx.synth_noise(R, 8, 3, 0.3, seed, False)
    a = W.scene_from_bits(bits, R, color, seed)
    if normals:
        a.brick_normal = vx.build_normals(a.brick_occ.reshape(-1, 16))
    return a, bits


def _same(a, b, color=True, normals=True):
    for f in FIELDS:
        np.testing.assert_array_equal(getattr(a, f), getattr(b, f), err_msg=f)
    assert tuple(a.world_min) == tuple(b.world_min) and tuple(a.world_max) == tuple(b.world_max)
    assert a.max_levels == b.max_levels and a.bricks_per_axis == b.bricks_per_axis
    if color:
        assert a.color_kind == b.color_kind
        np.testing.assert_array_equal(a.brick_color, b.brick_color)
    if normals:
        np.testing.assert_array_equal(a.brick_normal, b.brick_normal)


@pytest.mark.parametrize("color,normals", [("dxt1", True), ("rgba8", False), ("rgba8", True)])
def test_vxsc_round_trip(vx, tmp_path, color, normals):
    a, _ = _scene(vx, color, normals=normals)
    p = str(tmp_path / "s.vxsc")
    vx.cache_write(p, a)
    b = vx.cache_read(p)
    _same(a, b, True, normals)
    if not normals:
        assert b.brick_normal is None


def test_vxsc_rejects_damage(vx, tmp_path):
    a, _ = _scene(vx)
    p = tmp_path / "s.vxsc"
    vx.cache_write(str(p), a)
    raw = bytearray(p.read_bytes())
    for mutate in (lambda r: r.__setitem__(len(r) // 2, r[len(r) // 2] ^ 0x40),  # payload bit: checksum
                   lambda r: r.__delitem__(slice(len(r) - 100, len(r))),        # truncated
                   lambda r: r.__setitem__(0, r[0] ^ 1)):                       # magic
        r = bytearray(raw)
        mutate(r)
        q = tmp_path / "bad.vxsc"
        q.write_bytes(bytes(r))
        with pytest.raises(vx.VxError):
            vx.cache_read(str(q))
    with pytest.raises(vx.VxError):
        vx.cache_read(str(tmp_path / "missing.vxsc"))


def _ref_descriptors(a):
    """The arrays as the reference's 64-bit ChildDescriptor (SVOTypes.h:36-47)."""
    cp = a.nodes[0::2].astype(np.uint64)
    valid = (a.nodes[1::2] & 0xFF).astype(np.uint64)
    leaf = ((a.nodes[1::2] >> 8) & 0xFF).astype(np.uint64)
    assert np.all(cp < 0x8000)
    return cp | (valid << 16) | (leaf << 24) | (a.node_brick.astype(np.uint64) << 32)


def _pack_vsca(entries):
    """VoxelSceneCacher::SerializeToFile (VoxelSceneCacher.cpp:209-265), packed
    field by field: header, then per entry the key, CreateInfo, six vectors
    (u64 element count + raw data), OctreeConfig (260 bytes) and metadata."""
    out = [struct.pack("<III", 0x56534341, 1, len(entries))]
    for e in entries:
        a, (st, res, dens, seed) = e["arrays"], e["ci"]
        key = st
        for v in (res, int(np.float32(dens) * np.float32(100.0)), seed):
            key = (key * 31 + v) & 0xFFFFFFFFFFFFFFFF
        out.append(struct.pack("<QIIfI", key if not e.get("bad_key") else key + 1, st, res, dens, seed))
        esvo = _ref_descriptors(a).tobytes()
        B = a.brick_count
        occ_bits = np.unpackbits(a.brick_occ.reshape(B, 16).view(np.uint8), axis=1, bitorder="little")
        if "words" in e:  # per-voxel material words (0 for empty voxels)
            brick_data = np.ascontiguousarray(e["words"], np.uint32).tobytes()
        else:
            brick_data = np.where(occ_bits == 1, e.get("material", 1), 0).astype(np.uint32).tobytes()
        materials = np.zeros((e.get("n_materials", 64), 8), np.float32).tobytes()
        colors = a.brick_color.tobytes() if a.brick_color is not None and a.color_kind == 2 else b""
        normals = a.brick_normal.tobytes() if a.brick_normal is not None else b""
        grid = a.grid_lookup.astype(np.uint32).tobytes()
        for blob, elem in ((esvo, 1), (brick_data, 1), (materials, 32), (colors, 1), (normals, 1), (grid, 4)):
            out.append(struct.pack("<Q", len(blob) // elem) + blob)
        L = a.max_levels
        cfg = struct.pack("<8i", 22, L, 3, 8, 22 - L + 1, 22 - (L - 1 - (L - 3)), a.bricks_per_axis, 0)
        cfg += struct.pack("<4f", *a.world_min, 0.0) + struct.pack("<4f", *a.world_max, 0.0)
        cfg += np.diag(np.float32([10, 10, 10, 1])).tobytes() + np.diag(np.float32([0.1, 0.1, 0.1, 1])).tobytes()
        cfg += bytes(64) + struct.pack("<f", 10.0)
        assert len(cfg) == 260
        solid = int(occ_bits.sum())
        out.append(cfg + struct.pack("<5I", a.node_count, B, solid, res, st))
    return b"".join(out)


def test_vsca_reads_reference_layout(vx, vo, tmp_path):
    """Two entries packed in the reference's layout from the oracle's rebuild
    (descriptors in ChildDescriptor layout, brickData material ids 5 and 1,
    a 64-material table); entry 1 reads back as the oracle's arrays."""
    R = 64
    rng = np.random.default_rng(11)
    bits = (rng.integers(0, 2 ** 63, R * R, dtype=np.int64).view(np.uint64) &
            rng.integers(0, 2 ** 63, R * R, dtype=np.int64).view(np.uint64))
    o = vo.OracleScene.from_dense(bits, R, 6)
    ex = o.export()
    import vx_b200 as pkg
    a = pkg.SceneArrays((0.0, 0.0, 0.0), (64.0, 64.0, 64.0), 6, o.bricks_per_axis, ex["nodes"], ex["node_brick"],
                        ex["grid_lookup"], ex["brick_coord"], ex["brick_occ"], pkg.VX_COLOR_DXT1,
                        vx.synth_dxt1(ex["brick_coord"], 4), vo.brick_normals(ex["brick_occ"]))
    first, _ = _scene(vx, "dxt1", R=64, seed=9)
    p = tmp_path / "ref.vsca"
    p.write_bytes(_pack_vsca([{"arrays": first, "ci": (1, 64, 0.3, 9)},
                              {"arrays": a, "ci": (0, 64, 0.25, 42), "material": 5}]))
    b = vx.cache_read_vsca(str(p), 1)
    _same(a, b)
    c = vx.cache_read_vsca(str(p), 0)
    _same(first, c)
    with pytest.raises(vx.VxError):
        vx.cache_read_vsca(str(p), 2)
    q = tmp_path / "badkey.vsca"
    q.write_bytes(_pack_vsca([{"arrays": a, "ci": (0, 64, 0.25, 42), "bad_key": True}]))
    with pytest.raises(vx.VxError):
        vx.cache_read_vsca(str(q), 0)


def test_vsca_write_matches_reference_layout(vx, tmp_path):
    """The library's VSCA writer produces the bytes packed in the reference's
    order (empty material table), and reads back."""
    a, _ = _scene(vx, "dxt1", R=64, seed=5)
    p = tmp_path / "w.vsca"
    vx.cache_write_vsca(str(p), a, 2, 64, 0.5, 7)
    want = _pack_vsca([{"arrays": a, "ci": (2, 64, 0.5, 7), "n_materials": 0}])
    assert p.read_bytes() == want
    _same(a, vx.cache_read_vsca(str(p), 0))


def test_vsca_write_rejects_wide_child_pointers(vx, tmp_path):
    """ChildDescriptor's child pointer has 15 bits; a scene past 2^15
    descriptors is refused instead of truncated."""
    R = 256
    bits = np.full(R * R * (R // 64), 0x0101010101010101, np.uint64)  # every brick populated
    a = vx.build_dense(bits, R, 8)
    assert a.node_count > 0x8000
    with pytest.raises(vx.VxError):
        vx.cache_write_vsca(str(tmp_path / "big.vsca"), a, 0, R, 1.0, 0)
    vx.cache_write(str(tmp_path / "big.vxsc"), a)
    _same(a, vx.cache_read(str(tmp_path / "big.vxsc")), False, False)


def test_vxsc_header_sizes_checked_before_allocating(vx, tmp_path):
    """A header that promises 2^32 descriptors in a small file is rejected as a format error
    (no allocation of the promised size)."""
    import struct as st
    a, _ = _scene(vx)
    p = tmp_path / "s.vxsc"
    vx.cache_write(str(p), a)
    raw = bytearray(p.read_bytes())
    off = 8 + 40  # magic, version, vx_octree_config
    raw[off:off + 4] = st.pack("<I", 0xFFFFFFFF)
    q = tmp_path / "huge.vxsc"
    q.write_bytes(bytes(raw))
    with pytest.raises(vx.VxError):
        vx.cache_read(str(q))


def test_vsca_vector_sizes_checked(vx, tmp_path):
    a, _ = _scene(vx, "dxt1", R=64, seed=5)
    p = tmp_path / "w.vsca"
    vx.cache_write_vsca(str(p), a, 2, 64, 0.5, 7)
    raw = bytearray(p.read_bytes())
    import struct as st
    raw[12 + 8 + 16:12 + 8 + 16 + 8] = st.pack("<Q", 1 << 39)  # esvoNodes length
    q = tmp_path / "huge.vsca"
    q.write_bytes(bytes(raw))
    with pytest.raises(vx.VxError):
        vx.cache_read_vsca(str(q), 0)
