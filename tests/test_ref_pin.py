"""The oracle pinned to the reference's own code (CPU).

`make -C oracle ref` compiles the reference's LaineKarrasOctree::rebuild, castRay /
castRayWithLOD and brick DDA from its sources (SVO/src/SVORebuild.cpp, SVOTraversal.cpp,
SVOBrickDDA.cpp and their dependencies), with stand-ins for glm and gaia-ecs, which are not
installed here (oracle/ref_shim/).  These tests give the reference build and the oracle the
same voxels and the same rays and require the same results bit for bit: hit, t (tMin), tMax,
hit point, normal, scale, the hit entity's position, and the rebuilt ChildDescriptor words.

The stand-ins are the only code here that is not the reference's: glm's arithmetic as its
documentation defines it (the oracle makes the same substitution) and an entity store keyed
by the reference's own Morton keys.  Skipped where the reference build is absent (a machine
without the reference sources).
"""
import numpy as np
import pytest

import kat_cases as K
from conftest import load_oracle

load_oracle()  # puts oracle/ on the import path
import vx_ref as vr  # noqa: E402
pytestmark = pytest.mark.skipif(not vr.available(), reason="reference build absent (make -C oracle ref)")

FLT_MAX = 3.4028234663852886e38


def assert_same(ref, o, label):
    hit = ref["hit"].astype(bool)
    ohit = (o["flags"] & 1).astype(bool)
    bad = np.flatnonzero(hit != ohit)
    assert bad.size == 0, f"{label}: hit differs on {bad.size} rays, first {bad[0]}: ref={ref[bad[0]]} oracle={o[bad[0]]}"
    for f in ("t", "t_exit"):
        d = np.flatnonzero(hit & (ref[f].view(np.uint32) != o[f].view(np.uint32)))
        assert d.size == 0, f"{label}: {f} differs on {d.size} rays, first {d[0]}: ref={ref[d[0]]} oracle={o[d[0]]}"
    for f in ("hit_point", "normal"):
        d = np.flatnonzero(hit & np.any(ref[f].view(np.uint32) != o[f].view(np.uint32), axis=1))
        assert d.size == 0, f"{label}: {f} differs on {d.size} rays, first {d[0]}: ref={ref[d[0]]} oracle={o[d[0]]}"
    d = np.flatnonzero(hit & (ref["scale"] != o["scale"]))
    assert d.size == 0, f"{label}: scale differs on {d.size} rays"
    # the hit entity: a voxel hit carries the entity at the oracle's key; an LOD hit carries none
    vox = hit & (o["brick"] != 0xFFFFFFFF)
    d = np.flatnonzero(vox & np.any(ref["entity_pos"].astype(np.int64) != o["key"].astype(np.int64), axis=1))
    assert d.size == 0, f"{label}: entity differs on {d.size} rays, first {d[0]}: ref={ref[d[0]]} oracle={o[d[0]]}"
    assert np.all(ref["entity_pos"][hit & ~vox] == -1.0)
    return int(hit.sum())


def _oracle_ref_descriptors(o):
    e = o.export()
    cp = e["nodes"][0::2].astype(np.uint64)
    valid = (e["nodes"][1::2] & 0xFF).astype(np.uint64)
    leaf = ((e["nodes"][1::2] >> 8) & 0xFF).astype(np.uint64)
    return cp | (valid << 16) | (leaf << 24) | (e["node_brick"].astype(np.uint64) << 32)


def _unique_kat_scenes():
    seen = {}
    for c in K.CASES:
        seen.setdefault((tuple(map(tuple, c.voxels)), c.world_min, c.world_max, c.depth), []).append(c)
    return list(seen.values())


@pytest.mark.parametrize("case", K.CASES, ids=[c.name for c in K.CASES])
def test_kat_ray_equals_reference(vo, case):
    """Every ported castRay case, the nine the reference's own assertions reject included: the
    oracle's result is the reference code's result."""
    r = vr.RefOctree(case.voxels, case.world_min, case.world_max, case.depth)
    o = vo.OracleScene.from_positions(case.voxels, case.world_min, case.world_max, case.depth)
    ray = np.array([list(case.origin) + list(case.direction)], np.float32)
    assert_same(r.cast_rays(ray, case.tmin, case.tmax), o.cast_rays(ray, case.tmin, case.tmax), case.name)


@pytest.mark.parametrize("group", _unique_kat_scenes(), ids=lambda g: g[0].name)
def test_kat_scenes_random_rays_and_rebuild_equal_reference(vx, vo, group):
    from vx_b200 import workloads as W
    c = group[0]
    r = vr.RefOctree(c.voxels, c.world_min, c.world_max, c.depth)
    o = vo.OracleScene.from_positions(c.voxels, c.world_min, c.world_max, c.depth)
    if o.node_count < 0x8000:
        np.testing.assert_array_equal(r.descriptors(), _oracle_ref_descriptors(o))
    extent = float(np.max(np.asarray(c.world_max) - np.asarray(c.world_min)))
    rays = W.random_rays(3000, extent, seed=len(c.voxels), lo=-0.5, hi=1.5)
    rays[:, :3] += np.asarray(c.world_min, np.float32)
    for tmin, tmax in ((0.0, 100.0), (0.0, FLT_MAX), (2.5, 9.0)):
        assert_same(r.cast_rays(rays, tmin, tmax), o.cast_rays(rays, tmin, tmax), f"{c.name} t in [{tmin},{tmax}]")


@pytest.mark.parametrize("R,fill,seed,shell", [(64, 0.3, 3, False), (64, 0.1, 5, True), (128, 0.1, 7, True)])
def test_noise_scenes_equal_reference(vx, vo, R, fill, seed, shell):
    """Seeded noise scenes (the oracle's own generator), a camera from an empty voxel and random
    rays: every hit field and the rebuilt descriptors equal the reference's."""
    import workloads_ref as wr
    bits = wr.noise_bits(R, max(4, R // 8), 3, fill, seed, shell)
    r = vr.RefOctree.from_dense(bits, R, wr.levels_for(R))
    o = vo.OracleScene.from_dense(bits, R, wr.levels_for(R))
    if o.node_count < 0x8000:
        np.testing.assert_array_equal(r.descriptors(), _oracle_ref_descriptors(o))
    from vx_b200 import workloads as W
    cam = wr.empty_voxel_camera(bits, R, seed, 70.0, 64, 48) if not shell else \
        wr.look_camera([R / 2 + 0.5, R / 2 + 0.5, 1.5], [0, 0, 1], 60.0, 64, 48)
    rays = np.concatenate([vo.camera_rays(cam, 64, 48), W.random_rays(4000, R, seed=seed)])
    n = assert_same(r.cast_rays(rays), o.cast_rays(rays), f"noise {R}")
    assert n > 500


def test_lod_cut_equals_reference(vx, vo):
    """castRayWithLOD: the cut happens on the same cell with the same t and scale."""
    import workloads_ref as wr
    bits = wr.noise_bits(64, 8, 3, 0.3, 9, False)
    r = vr.RefOctree.from_dense(bits, 64, 6)
    o = vo.OracleScene.from_dense(bits, 64, 6)
    from vx_b200 import workloads as W
    rays = W.random_rays(4000, 64, seed=19)
    for lod in ((0.0, 0.01), (0.5, 0.05), (0.0, 0.2)):
        ref = r.cast_rays(rays, lod=lod)
        assert_same(ref, o.cast_rays_lod(rays, lod), f"lod {lod}")


@pytest.mark.parametrize("R,fill,seed", [(64, 0.3, 4), (64, 0.6, 6)])
def test_rebuild_payloads_equal_reference(vx, vo, R, fill, seed):
    """The compression phase of the reference's rebuild (SVORebuild.cpp:609-722) on voxels with
    Material ids: its DXT normal payload equals vx_build_normals (and the oracle's), its DXT1
    colour payload equals vx_build_dxt1 over vx_material_rgb of the words (MaterialIdToColor),
    and its brickMaterialData equals the words in the library's brick order."""
    import workloads_ref as wr
    bits = wr.noise_bits(R, 8, 3, fill, seed, False)
    pool = np.array([1, 2, 3, 7, 10, 20, 30, 33, 35, 39, 40, 50, 61, 77, 150, 255], np.uint32)
    mat_of = lambda x, y, z: pool[(x * 7 + y * 13 + z * 29) % pool.size]  # noqa: E731
    r = vr.RefOctree.from_dense(bits, R, wr.levels_for(R), mat_of)
    col, nrm, mat = r.payloads()
    a = vx.build_dense(bits, R, wr.levels_for(R))
    B = a.brick_count
    assert col.size == B * 32
    # material words in brick order, from the brick coordinates
    v = np.arange(512)
    c = a.brick_coord.astype(np.int64)
    bx, by, bz = (c & 0x3FF) * 8, ((c >> 10) & 0x3FF) * 8, ((c >> 20) & 0x3FF) * 8
    x, y, z = bx[:, None] + (v & 7), by[:, None] + ((v >> 3) & 7), bz[:, None] + (v >> 6)
    occ = np.unpackbits(a.brick_occ.reshape(B, 16).view(np.uint8), axis=1, bitorder="little").astype(bool)
    words = np.where(occ, mat_of(x, y, z), 0).astype(np.uint32).reshape(-1)
    np.testing.assert_array_equal(mat, words)
    np.testing.assert_array_equal(nrm, vx.build_normals(a.brick_occ.reshape(-1, 16)))
    np.testing.assert_array_equal(nrm, vo.brick_normals(a.brick_occ))
    rgb = vx.material_rgb(words)
    np.testing.assert_array_equal(col, vx.build_dxt1(rgb.reshape(-1, 512, 3), a.brick_occ))
    np.testing.assert_array_equal(col, vo.brick_dxt1(rgb.reshape(-1), a.brick_occ))
