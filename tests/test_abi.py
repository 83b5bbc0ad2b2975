"""The C ABI library loads and exports every entry point include/vx.h declares;
argument validation runs on the host without a GPU (CPU only)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "vx.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|int32_t|const char\*)\s+(vx_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ["vx_scene_create", "vx_scene_destroy", "vx_cast_rays", "vx_cast_rays_host", "vx_render",
              "vx_build_dense", "vx_last_error_string"]:
        assert n in names


def test_library_exports_every_declared_symbol(vx):
    L = vx.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_abi_version(vx):
    assert vx.lib().vx_abi_version() == 2


def test_struct_sizes(vx):
    assert vx.HIT_DTYPE.itemsize == 16
    assert C.sizeof(vx.CameraPC) == 64
    assert C.sizeof(vx._SceneDesc) == 112


def _desc(vx, **over):
    d = vx._SceneDesc()
    d.config.world_min[:] = [0, 0, 0]
    d.config.world_max[:] = [64, 64, 64]
    d.config.max_levels = 6
    d.config.brick_depth = 3
    d.config.bricks_per_axis = 8
    for k, v in over.items():
        if k in ("max_levels", "brick_depth", "bricks_per_axis"):
            setattr(d.config, k, v)
        else:
            setattr(d, k, v)
    return d


def test_scene_create_rejects_bad_config_on_host(vx):
    grid = np.full(512, 0xFFFFFFFF, np.uint32)
    h = C.c_void_p()
    for over, msg in [(dict(brick_depth=4), "brick_depth"), (dict(max_levels=0), "max_levels"),
                      (dict(bricks_per_axis=7), "bricks_per_axis"), (dict(color_kind=7), "color_kind")]:
        d = _desc(vx, grid_lookup=grid.ctypes.data, **over)
        assert vx.lib().vx_scene_create(C.byref(d), C.byref(h)) == -1
        assert msg in vx.lib().vx_last_error_string().decode()
    bad = grid.copy()
    bad[3] = 5  # brick index with no bricks
    d = _desc(vx, grid_lookup=bad.ctypes.data)
    assert vx.lib().vx_scene_create(C.byref(d), C.byref(h)) == -1
    assert "grid_lookup[3]" in vx.lib().vx_last_error_string().decode()


def test_null_arguments(vx):
    L = vx.lib()
    assert L.vx_scene_create(None, None) == -1
    assert L.vx_cast_rays(None, None, 1, 0.0, 1.0, None, None, None, None) == -1
    assert L.vx_render(None, None, 1, 1, None, None, None, None) == -1
    assert L.vx_build_dense(None, 64, 6, None) == -1
    assert L.vx_batch_capture_frame(None, None, None, 1, None, None, None, None, 0, None) == -1
    assert L.vx_batch_capture_frame_compact(None, None, None, 1, None, None, None, 0, None) == -1
    assert b"capture_frame_compact" in L.vx_last_error_string()
    assert L.vx_batch_launch_frame(None, None) == -1
    assert L.vx_scene_destroy(None) == 0


def test_error_string_is_thread_local(vx):
    import threading
    L = vx.lib()
    L.vx_scene_create(None, None)
    seen = []
    t = threading.Thread(target=lambda: seen.append(L.vx_last_error_string()))
    t.start()
    t.join()
    assert seen == [b""]
    assert L.vx_last_error_string() != b""


def test_camera_rays_host(vx):
    pc = vx.CameraPC.make([1, 2, 3], [0, 0, 1], [0, 1, 0], [-1, 0, 0], 60.0, 1.0)
    r = vx.camera_rays(pc, 4, 2)
    assert r.shape == (8, 6)
    assert np.all(r[:, :3] == np.float32([1, 2, 3]))
    n = np.linalg.norm(r[:, 3:].astype(np.float64), axis=1)
    assert np.all(np.abs(n - 1) < 1e-6)
    assert r[0, 4] > 0 and r[-1, 4] < 0  # row 0 is the top of the image


def test_default_build_compiles_no_bounds_checks(vx):
    en = C.c_int32(-1)
    assert vx.lib().vx_bounds_checks(C.byref(en), None) == 0
    assert en.value == 0
