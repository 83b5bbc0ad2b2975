"""CUDA kernels against the CPU oracle, bit for bit (needs a B200).

Hit voxel, brick and node indices, the hit flags and the DXT texel must be
identical; t is compared as raw binary32 bits (0 ulp, inside the 2-ulp bound
the specification allows).  Every call goes through the C ABI (libvx.so).
"""
import numpy as np
import pytest

import kat_cases as K

pytestmark = pytest.mark.gpu

FLT_MAX = 3.4028234663852886e38


def scene_from_oracle(vx, o, case_or_bounds, levels):
    e = o.export()
    wmin, wmax = case_or_bounds
    return vx.SceneArrays(tuple(float(v) for v in wmin), tuple(float(v) for v in wmax), levels, o.bricks_per_axis,
                          e["nodes"], e["node_brick"], e["grid_lookup"], e["brick_coord"], e["brick_occ"])


def gpu_cast(vx, scene, rays, tmin=0.0, tmax=FLT_MAX, with_counters=True):
    import torch
    s = scene if isinstance(scene, vx.Scene) else vx.Scene(scene)
    n = rays.shape[0]
    r = torch.from_numpy(np.ascontiguousarray(rays, np.float32)).cuda()
    hits = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    cw = s.color_width()
    color = None
    if cw:
        color = torch.zeros((n, cw), dtype=torch.int32 if cw == 1 else torch.float32, device="cuda")
    counters = torch.zeros((n, 4), dtype=torch.int32, device="cuda") if with_counters else None
    s.cast_rays_dev(r, hits, color, counters, tmin, tmax)
    torch.cuda.synchronize()
    h = hits.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1)
    c = None if color is None else color.cpu().numpy()
    cnt = None if counters is None else counters.cpu().numpy().view(vx.COUNTER_DTYPE).reshape(-1)
    return h, c, cnt


def assert_hits_equal(g, o, cnt=None, label=""):
    mism = {}
    mism["flags"] = np.flatnonzero(g["flags"].astype(np.uint32) != o["flags"])
    hit = (o["flags"] & 1).astype(bool)
    mism["t"] = np.flatnonzero(hit & (g["t"].view(np.uint32) != o["t"].view(np.uint32)))
    mism["brick"] = np.flatnonzero(g["brick"] != o["brick"])
    mism["node"] = np.flatnonzero(g["node"] != o["node"])
    mism["voxel"] = np.flatnonzero(g["voxel"].astype(np.uint32) != o["voxel"])
    mism["scale"] = np.flatnonzero(g["scale"].astype(np.int32) != o["scale"])
    if cnt is not None:
        mism["iters"] = np.flatnonzero(cnt["iters"].astype(np.uint32) != o["iters"])
        mism["grid_reads"] = np.flatnonzero(cnt["grid_reads"].astype(np.uint32) != o["grid_reads"])
        mism["dda_steps"] = np.flatnonzero(cnt["dda_steps"].astype(np.uint32) != o["dda_steps"])
    bad = {k: v for k, v in mism.items() if v.size}
    if bad:
        k, idx = next(iter(bad.items()))
        i = int(idx[0])
        raise AssertionError(f"{label}: mismatches {({k: v.size for k, v in bad.items()})}; first ray {i}: "
                             f"gpu={g[i]} oracle={o[i]}")


def _unique_kat_scenes():
    seen = {}
    for c in K.CASES:
        key = (tuple(c.voxels), c.world_min, c.world_max, c.depth)
        seen.setdefault(key, []).append(c)
    return list(seen.values())


@pytest.mark.parametrize("group", _unique_kat_scenes(), ids=lambda g: g[0].name)
def test_kat_scenes_bit_exact(vx, vo, cuda, group):
    from vx_b200 import workloads as W
    c0 = group[0]
    o = vo.OracleScene.from_positions(c0.voxels, c0.world_min, c0.world_max, c0.depth)
    scene = scene_from_oracle(vx, o, (c0.world_min, c0.world_max), c0.depth)
    extent = float(np.max(np.asarray(c0.world_max) - np.asarray(c0.world_min)))
    rays = W.random_rays(4000, extent, seed=len(c0.voxels), lo=-0.5, hi=1.5)
    rays[:, :3] += np.asarray(c0.world_min, np.float32)
    kat = np.array([list(c.origin) + list(c.direction) for c in group], np.float32)
    rays = np.concatenate([kat, rays])
    g, _, cnt = gpu_cast(vx, scene, rays, 0.0, 100.0)
    assert_hits_equal(g, o.cast_rays(rays, 0.0, 100.0), cnt, c0.name)


@pytest.mark.parametrize("R", [64, 128])
def test_noise_scene_rgba8_bit_exact(vx, vo, cuda, R):
    from vx_b200 import workloads as W
    wl = W.config1(R=R, width=128, height=128, seed=R)
    o = vo.OracleScene.from_dense(wl.bits, R, wl.scene.max_levels)
    rays = np.concatenate([wl.rays(), W.random_rays(20000, R, seed=3)])
    g, col, cnt = gpu_cast(vx, wl.scene, rays)
    oh = o.cast_rays(rays)
    assert_hits_equal(g, oh, cnt, wl.name)
    hit = (oh["flags"] & 1).astype(bool)
    assert hit.mean() > 0.1
    want = np.zeros(rays.shape[0], np.uint32)
    want[hit] = wl.scene.brick_color[oh["brick"][hit].astype(np.int64) * 512 + oh["voxel"][hit]]
    np.testing.assert_array_equal(col[:, 0].view(np.uint32), want)


@pytest.mark.parametrize("L", [16, 20, 23])
def test_deep_scene_bit_exact(vx, vo, cuda, L):
    """max_levels 16-23 over a 64^3 grid: the per-thread stacks grow to two words per level
    plus the cycle-detection slots, 51-64 KiB of shared memory for the batched kernel's
    256-thread blocks (above the 48 KiB a launch gets without opting in).  Plain cast,
    render, batched cast and the adjoint forward run and stay bit-exact."""
    import torch
    from vx_b200 import workloads as W
    bits = vx.synth_noise(64, 8, 3, 0.5, 41, False)
    a = W.scene_from_bits(bits, 64, "rgba8", 41, max_levels=L)
    o = vo.OracleScene.from_dense(bits, 64, L)
    cam = W.empty_voxel_camera(bits, 64, 41, 70.0, 64, 48)
    cam_rays = vx.camera_rays(cam, 64, 48)
    rays = np.concatenate([cam_rays, W.random_rays(8000, 64, seed=43)])
    s = vx.Scene(a)
    g, col, cnt = gpu_cast(vx, s, rays)
    oh = o.cast_rays(rays)
    assert_hits_equal(g, oh, cnt, f"deep L={L}")
    assert (oh["flags"] & 1).mean() > 0.1
    n = 64 * 48
    want = o.cast_rays(cam_rays)
    img = torch.zeros(n, dtype=torch.int32, device="cuda")
    hits = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    s.render_dev(cam, 64, 48, img, hits)
    torch.cuda.synchronize()
    assert_hits_equal(hits.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1), want, None, "render")
    r = torch.from_numpy(rays).cuda()
    bh = torch.zeros((rays.shape[0], 4), dtype=torch.int32, device="cuda")
    batch = vx.Batch([s])
    batch.set_tuning(256, 32, 1, 0)
    batch.cast(r, torch.tensor([0, rays.shape[0]], dtype=torch.int32, device="cuda"), bh)
    torch.cuda.synchronize()
    assert_hits_equal(bh.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1), oh, None, "batched")
    batch.close()
    attr = torch.rand(a.brick_count * 512 * 3, device="cuda")
    image = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    rec = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    vx.diff_forward(s, cam, 64, 48, 0, attr, None, image, rec)
    torch.cuda.synchronize()
    assert_hits_equal(rec.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1), want, None, "adjoint forward")


def test_dxt_scene_texels_bit_exact(vx, vo, cuda):
    from vx_b200 import workloads as W
    wl = W.config2(R=128, width=160, height=90, seed=5)
    o = vo.OracleScene.from_dense(wl.bits, 128, wl.scene.max_levels)
    rays = np.concatenate([wl.rays(), W.random_rays(20000, 128, seed=9)])
    g, col, cnt = gpu_cast(vx, wl.scene, rays)
    oh = o.cast_rays(rays)
    assert_hits_equal(g, oh, cnt, wl.name)
    hit = np.flatnonzero(oh["flags"] & 1)
    assert hit.size > 1000
    for i in hit[:: max(1, hit.size // 3000)]:
        want = vo.hit_texel_dxt(wl.scene.brick_color, int(oh["brick"][i]), int(oh["voxel"][i]))
        np.testing.assert_array_equal(col[i].view(np.uint32), want.view(np.uint32))
    assert np.all(col[(oh["flags"] & 1) == 0] == 0)


def test_config1_full_size_bit_exact(vx, vo, cuda):
    """cfg1 at its full size: 256^3, 512x512 primary rays, every ray checked."""
    from vx_b200 import workloads as W
    wl = W.config1()
    o = vo.OracleScene.from_dense(wl.bits, 256, 8)
    rays = wl.rays()
    g, col, cnt = gpu_cast(vx, wl.scene, rays)
    oh = o.cast_rays(rays)
    assert_hits_equal(g, oh, cnt, wl.name)
    assert (oh["flags"] & 1).mean() > 0.2


def test_t_range_clipping(vx, vo, cuda):
    from vx_b200 import workloads as W
    wl = W.config1(R=64, width=64, height=64, seed=2)
    o = vo.OracleScene.from_dense(wl.bits, 64, wl.scene.max_levels)
    rays = W.random_rays(5000, 64, seed=4)
    s = vx.Scene(wl.scene)
    for tmin, tmax in [(0.0, 10.0), (5.0, 40.0), (30.0, 31.0), (-5.0, 1e9), (50.0, 20.0)]:
        g, _, cnt = gpu_cast(vx, s, rays, tmin, tmax)
        assert_hits_equal(g, o.cast_rays(rays, tmin, tmax), cnt, f"t in [{tmin},{tmax}]")


def test_degenerate_rays(vx, vo, cuda):
    from vx_b200 import workloads as W
    wl = W.config1(R=64, width=8, height=8, seed=3)
    o = vo.OracleScene.from_dense(wl.bits, 64, wl.scene.max_levels)
    nan, inf = np.float32(np.nan), np.float32(np.inf)
    rays = np.array([[32, 32, 32, 0, 0, 0], [32, 32, 32, nan, 1, 0], [nan, 1, 1, 1, 0, 0],
                     [inf, 1, 1, -1, 0, 0], [32, 32, 32, 1e-30, 0, 0], [32, 32, 32, 0, 0, -1e-12],
                     [-10, 32.5, 32.5, 1, 0, 0], [0, 0, 0, 1, 1, 1], [64, 64, 64, -1, -1, -1],
                     [32, 32, 32, 1e-6, 1e-6, 1], [1.0, 1.0, 1.0, -1, 0, 0], [32, 32, -1, 0, 0, 1]],
                    np.float32)
    g, _, cnt = gpu_cast(vx, wl.scene, rays)
    oh = o.cast_rays(rays)
    assert_hits_equal(g, oh, cnt, "degenerate")
    assert oh["flags"][0] & vx.VX_RAY_INVALID and oh["flags"][1] & vx.VX_RAY_INVALID


def test_empty_scene_rays_invalid(vx, cuda):
    a = vx.build_dense(np.zeros(64 * 64, np.uint64), 64, 6)
    g, _, _ = gpu_cast(vx, a, np.array([[1, 1, 1, 1, 0, 0]], np.float32))
    assert g["flags"][0] == vx.VX_RAY_INVALID and g["brick"][0] == 0xFFFFFFFF


def test_host_entry_point_matches_device(vx, cuda):
    from vx_b200 import workloads as W
    wl = W.config2(R=64, width=64, height=48, seed=7)
    s = vx.Scene(wl.scene)
    rays = wl.rays()
    gd, cd, _ = gpu_cast(vx, s, rays, with_counters=False)
    gh, ch = s.cast_rays_host(rays)
    np.testing.assert_array_equal(gd.view(np.uint8), gh.view(np.uint8))
    np.testing.assert_array_equal(cd.view(np.uint32), ch.view(np.uint32))


@pytest.mark.parametrize("n", [1048575, 1048576, 2500001])
def test_host_entry_point_pipelined_chunks(vx, cuda, n):
    """Large host casts run as overlapped chunks; results equal the device call."""
    import torch
    from vx_b200 import workloads as W
    wl = W.config2(R=128, width=8, height=8, seed=17)
    s = vx.Scene(wl.scene)
    rays = W.random_rays(n, 128, seed=n)
    gd, cd, _ = gpu_cast(vx, s, rays, with_counters=False)
    pinned = torch.from_numpy(rays).pin_memory()
    gh, ch = s.cast_rays_host(pinned.numpy())
    np.testing.assert_array_equal(gd.view(np.uint8), gh.view(np.uint8))
    np.testing.assert_array_equal(cd.view(np.uint32), ch.view(np.uint32))


def test_camera_rays_device_equal_oracle(vx, vo, cuda):
    """vx_camera_rays_dev equals the oracle's restatement of getRayDir (RayGeneration.glsl:61-71)
    and the shader's pixel uv (VoxelRayMarch.comp:453-455) bit for bit, as does the host form."""
    import ctypes as C
    import torch
    from vx_b200 import workloads as W
    for pos, d, fov, w, h in [([10.5, 20.25, -3.0], [0.3, -0.2, 1.0], 70.0, 333, 177),
                              ([512.5, 100.0, 3.0], [-0.7, 0.1, 0.2], 60.0, 1920, 1080),
                              ([1.0, 2.0, 3.0], [0.0, -1.0, 0.0], 90.0, 64, 64)]:
        pc = W.look_camera(pos, d, fov, w, h)
        want = vo.camera_rays(pc, w, h)
        dev = torch.zeros((w * h, 6), dtype=torch.float32, device="cuda")
        vx.check(vx.lib().vx_camera_rays_dev(C.byref(pc), w, h, C.c_void_p(dev.data_ptr()), None))
        torch.cuda.synchronize()
        np.testing.assert_array_equal(dev.cpu().numpy().view(np.uint32), want.view(np.uint32))
        np.testing.assert_array_equal(vx.camera_rays(pc, w, h).view(np.uint32), want.view(np.uint32))


def test_render_matches_oracle_shading(vx, vo, cuda):
    import torch
    from vx_b200 import workloads as W
    wl = W.config1(R=128, width=96, height=80, seed=8)
    s = vx.Scene(wl.scene)
    n = wl.width * wl.height
    img = torch.zeros(n, dtype=torch.int32, device="cuda")
    hits = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    s.render_dev(wl.camera, wl.width, wl.height, img, hits)
    torch.cuda.synchronize()
    g = hits.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1)
    image = img.cpu().numpy().view(np.uint32)
    o = vo.OracleScene.from_dense(wl.bits, 128, wl.scene.max_levels)
    # the render kernel's in-kernel rays are checked through its hits: the oracle casts the rays of
    # its own restatement of the shader's ray generation
    rays, uv_y = vo.camera_rays(wl.camera, wl.width, wl.height, with_uv_y=True)
    oh = o.cast_rays(rays)
    assert_hits_equal(g, oh, None, "render hits")
    for i in range(n):
        hit = bool(oh["flags"][i] & 1)
        if hit:
            c = int(wl.scene.brick_color[int(oh["brick"][i]) * 512 + int(oh["voxel"][i])])
            col = np.array([c & 255, (c >> 8) & 255, (c >> 16) & 255], np.float32) / np.float32(255.0)
        else:
            col = np.zeros(3, np.float32)
        want = vo.shade(col, hit, (int(oh["flags"][i]) >> 1) & 3, bool(oh["flags"][i] & 8), float(uv_y[i]))
        assert image[i] == want, (i, hex(image[i]), hex(want))


def test_cornell_box_wall_colours(vx, vo, cuda):
    """CornellBoxTest (test_cornell_box.cpp:186-233, 290-322): the hit voxel's colour is its
    wall's (red left, grey floor), read through the RGBA8 colour output of the cast."""
    import math
    import torch
    cb = K.cornell_box_voxels()
    keys = {}
    for p, col in cb:  # later voxels at the same integer key replace earlier ones
        k = tuple(int(math.floor(np.float32(c) + np.float32(1e-5))) for c in p)
        keys[k] = col
    o = vo.OracleScene.from_positions([p for p, _ in cb], *K.CB_BOUNDS, 8)
    a = scene_from_oracle(vx, o, K.CB_BOUNDS, 8)
    B = a.brick_count
    rgba = np.zeros(B * 512, np.uint32)
    for b in range(B):
        c = int(a.brick_coord[b])
        bx, by, bz = (c & 0x3FF) * 8, ((c >> 10) & 0x3FF) * 8, ((c >> 20) & 0x3FF) * 8
        for v in range(512):
            col = keys.get((bx + (v & 7), by + ((v >> 3) & 7), bz + (v >> 6)))
            if col is not None:
                r, g, bl = (int(np.float32(x) * 255 + 0.5) for x in col)
                rgba[b * 512 + v] = r | (g << 8) | (bl << 16) | (255 << 24)
    a.color_kind, a.brick_color = vx.VX_COLOR_RGBA8, rgba
    rays = np.array([[5, 5, 5, 0, -1, 0], [5, 5, 5, -1, 0, 0]], np.float32)
    g, col, _ = gpu_cast(vx, a, rays, 0.0, 100.0)
    assert_hits_equal(g, o.cast_rays(rays, 0.0, 100.0), None, "cornell")
    assert g["flags"][0] & 1 and g["flags"][1] & 1
    c0, c1 = int(col[0, 0]) & 0xFFFFFFFF, int(col[1, 0]) & 0xFFFFFFFF
    assert (c0 & 255) == (c0 >> 8) & 255 == 204          # floor: grey 0.8
    assert (c1 & 255) > 127 and ((c1 >> 8) & 255) < 77   # left wall: red
