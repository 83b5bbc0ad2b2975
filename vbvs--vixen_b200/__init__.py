"""Python binding of libvx (include/vx.h): B200-native ESVO voxel ray casting.

Mirrors the reference's query interface for the ray-casting path:
`CudaOctree.castRay(origin, direction, tMin, tMax)` returns a `RayHit` with the
fields of ISVOStructure::RayHit (SVO/include/ISVOStructure.h:101-112), and
`castRays` casts a whole batch on the GPU.  `render` is the compute-dispatch
node's frame (RenderGraph/src/Nodes/ComputeDispatchNode.cpp:249-317) with the
swapchain image replaced by a device buffer.

Every call goes through libvx.so; there is no CPU fallback.  Importing this
module fails loudly when the library has not been built.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# VX_LIBRARY=checked loads the bounds-checked build (vx_bounds_checks).
LIB_PATH = os.path.join(_HERE, "libvx_checked.so" if os.environ.get("VX_LIBRARY") == "checked" else "libvx.so")

VX_OK = 0
VX_HIT_HIT = 0x01
VX_HIT_NORMAL_NEG = 0x08
VX_RAY_ITER_CAP = 0x40
VX_RAY_INVALID = 0x80
VX_COLOR_NONE, VX_COLOR_RGBA8, VX_COLOR_DXT1, VX_COLOR_MATERIAL = 0, 1, 2, 3
FLT_MAX = 3.4028234663852886e38
NONE = 0xFFFFFFFF

HIT_DTYPE = np.dtype([("t", "<f4"), ("brick", "<u4"), ("node", "<u4"), ("voxel", "<u2"),
                      ("flags", "u1"), ("scale", "u1")])
RAY_DTYPE = np.dtype([("o", "<f4", 3), ("d", "<f4", 3)])
COUNTER_DTYPE = np.dtype([("iters", "<u2"), ("grid_reads", "<u2"), ("dda_steps", "<u4"), ("run_iters", "<u2"),
                          ("run_grid_reads", "<u2"), ("run_dda_steps", "<u4")])


class VxError(RuntimeError):
    """A libvx call returned an error status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"libvx error {status}: {message}")
        self.status = status


class _Config(C.Structure):
    _fields_ = [("world_min", C.c_float * 3), ("world_max", C.c_float * 3), ("max_levels", C.c_int32),
                ("brick_depth", C.c_int32), ("bricks_per_axis", C.c_int32), ("reserved", C.c_int32)]


class _SceneDesc(C.Structure):
    _fields_ = [("config", _Config), ("nodes", C.c_void_p), ("node_count", C.c_uint32),
                ("brick_count", C.c_uint32), ("node_brick", C.c_void_p), ("grid_lookup", C.c_void_p),
                ("brick_coord", C.c_void_p), ("brick_occ", C.c_void_p), ("color_kind", C.c_int32),
                ("brick_color", C.c_void_p), ("brick_normal", C.c_void_p)]


class CameraPC(C.Structure):
    """PushConstants of shaders/VoxelRayMarch.comp:85-94 (64 bytes)."""
    _fields_ = [("camera_pos", C.c_float * 3), ("time", C.c_float), ("camera_dir", C.c_float * 3),
                ("fov", C.c_float), ("camera_up", C.c_float * 3), ("aspect", C.c_float),
                ("camera_right", C.c_float * 3), ("debug_mode", C.c_int32)]

    @classmethod
    def make(cls, pos, direction, up, right, fov_deg, aspect):
        pc = cls()
        pc.camera_pos[:] = [float(v) for v in pos]
        pc.camera_dir[:] = [float(v) for v in direction]
        pc.camera_up[:] = [float(v) for v in up]
        pc.camera_right[:] = [float(v) for v in right]
        pc.fov = float(fov_deg)
        pc.aspect = float(aspect)
        return pc


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libvx.so is not built ({LIB_PATH}); run __graft_entry__.build() or make -C vbvs--vixen_b200")
    L = C.CDLL(LIB_PATH)
    vp, u32, i32, u64, f32 = C.c_void_p, C.c_uint32, C.c_int32, C.c_uint64, C.c_float
    sig = {
        "vx_abi_version": (i32, []),
        "vx_last_error_string": (C.c_char_p, []),
        "vx_scene_create": (C.c_int, [vp, vp]),
        "vx_scene_destroy": (C.c_int, [vp]),
        "vx_scene_device_bytes": (C.c_int, [vp, vp]),
        "vx_cast_rays": (C.c_int, [vp, vp, u32, f32, f32, vp, vp, vp, vp]),
        "vx_cast_rays_host": (C.c_int, [vp, vp, u32, f32, f32, vp, vp, vp]),
        "vx_cast_rays_lod": (C.c_int, [vp, vp, u32, f32, f32, vp, vp, vp, vp, vp]),
        "vx_cast_rays_host_lod": (C.c_int, [vp, vp, u32, f32, f32, vp, vp, vp, vp]),
        "vx_lod_from_camera": (C.c_int, [f32, C.c_int32, f32, vp]),
        "vx_lod_with_bias": (C.c_int, [vp, f32, vp]),
        "vx_build_normals": (C.c_int, [vp, u32, vp]),
        "vx_build_normals_dev": (C.c_int, [vp, u32, vp, vp]),
        "vx_hit_normals": (C.c_int, [vp, vp, u32, vp, vp]),
        "vx_bounds_checks": (C.c_int, [vp, vp]),
        "vx_diff_forward_views": (C.c_int, [vp, vp, u32, u32, u32, i32, vp, vp, vp, vp, vp]),
        "vx_build_dxt1": (C.c_int, [vp, vp, u32, vp]),
        "vx_build_dxt1_dev": (C.c_int, [vp, vp, u32, vp, vp]),
        "vx_scene_info_get": (C.c_int, [vp, vp]),
        "vx_scene_download": (C.c_int, [vp, vp, vp, vp, vp, vp, vp, vp]),
        "vx_scene_create_dense_dev": (C.c_int, [vp, u32, i32, i32, u64, i32, vp, vp]),
        "vx_cache_write": (C.c_int, [C.c_char_p, vp]),
        "vx_cache_read": (C.c_int, [C.c_char_p, vp]),
        "vx_cache_write_vsca": (C.c_int, [C.c_char_p, vp, u32, u32, f32, u32]),
        "vx_cache_read_vsca": (C.c_int, [C.c_char_p, u32, vp]),
        "vx_cache_desc": (C.c_int, [vp, vp]),
        "vx_cache_desc_materials": (C.c_int, [vp, vp]),
        "vx_material_rgb": (C.c_int, [vp, u64, vp]),
        "vx_material_rgb_dev": (C.c_int, [vp, u64, vp, vp]),
        "vx_cache_free": (C.c_int, [vp]),
        "vx_scene_save": (C.c_int, [vp, C.c_char_p]),
        "vx_scene_load": (C.c_int, [C.c_char_p, vp]),
        "vx_render": (C.c_int, [vp, vp, u32, u32, vp, vp, vp, vp]),
        "vx_camera_rays": (C.c_int, [vp, u32, u32, vp]),
        "vx_camera_rays_dev": (C.c_int, [vp, u32, u32, vp, vp]),
        "vx_build_dense": (C.c_int, [vp, u32, i32, vp]),
        "vx_build_desc": (C.c_int, [vp, vp]),
        "vx_build_free": (C.c_int, [vp]),
        "vx_nodes_from_reference": (C.c_int, [vp, u32, vp, vp]),
        "vx_synth_noise": (C.c_int, [u32, u32, u32, f32, u64, i32, vp]),
        "vx_synth_noise_dev": (C.c_int, [u32, u32, u32, f32, u64, i32, vp, vp]),
        "vx_synth_urban": (C.c_int, [u32, u32, u32, u64, vp]),
        "vx_synth_rgba8": (C.c_int, [vp, u32, u64, vp]),
        "vx_synth_dxt1": (C.c_int, [vp, u32, u64, vp]),
        "vx_batch_create": (C.c_int, [vp, u32, vp]),
        "vx_batch_destroy": (C.c_int, [vp]),
        "vx_batch_set_tuning": (C.c_int, [vp, vp]),
        "vx_batch_get_tuning": (C.c_int, [vp, vp]),
        "vx_cast_batch": (C.c_int, [vp, vp, vp, u32, f32, f32, vp, vp, vp]),
        "vx_batch_autotune": (C.c_int, [vp, vp, vp, u32, vp, vp, vp, vp]),
        "vx_spawn_bounce_rays": (C.c_int, [vp, vp, u32, u64, vp, vp]),
        "vx_spawn_shadow_rays": (C.c_int, [vp, vp, u32, vp, vp, vp]),
        "vx_bounce_table": (C.c_int, [vp]),
        "vx_batch_capture_frame": (C.c_int, [vp, vp, vp, u32, vp, vp, vp, vp, u64, vp]),
        "vx_batch_capture_frame_compact": (C.c_int, [vp, vp, vp, u32, vp, vp, vp, u64, vp]),
        "vx_batch_capture_frame_parts": (C.c_int, [vp, vp, vp, u32, vp, vp, vp, u64, u32, vp]),
        "vx_cast_shadow_rays": (C.c_int, [vp, vp, vp, u32, vp, C.c_float, C.c_float, vp, vp]),
        "vx_batch_launch_frame": (C.c_int, [vp, vp]),
        "vx_batch_launch_frame_host": (C.c_int, [vp, vp, vp, vp, vp]),
        "vx_batch_frame_compaction": (C.c_int, [vp, vp, vp, vp, vp]),
        "vx_batch_set_bounce_tuning": (C.c_int, [vp, vp]),
        "vx_cast_batch_noalloc": (C.c_int, [vp, u32, vp, vp, u32, f32, f32, vp, vp]),
        "vx_diff_forward": (C.c_int, [vp, vp, u32, u32, i32, vp, vp, vp, vp, vp]),
        "vx_diff_backward": (C.c_int, [u32, i32, vp, vp, vp, vp, vp, vp, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(status: int) -> None:
    if status != VX_OK:
        raise VxError(status, lib().vx_last_error_string().decode(errors="replace"))


def _p(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data_as(C.c_void_p)
    return C.c_void_p(int(a.data_ptr()))  # torch tensor


# ---------------------------------------------------------------------------
# Synthetic inputs and the host builder
# ---------------------------------------------------------------------------

def synth_noise(R: int, spacing: int, octaves: int, fill: float, seed: int, shell: bool) -> np.ndarray:
    bits = np.zeros(R * R * (R // 64), np.uint64)
    check(lib().vx_synth_noise(R, spacing, octaves, float(fill), seed, int(shell), _p(bits)))
    return bits


def synth_noise_dev(R: int, spacing: int, octaves: int, fill: float, seed: int, shell: bool, out=None):
    """vx_synth_noise on the current CUDA device; returns a uint64 CUDA tensor (as int64)."""
    import torch
    if out is None:
        out = torch.empty(R * R * (R // 64), dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    check(lib().vx_synth_noise_dev(R, spacing, octaves, float(fill), seed, int(shell), _p(out), C.c_void_p(s)))
    return out


def synth_urban(R: int, hmin: int, hmax: int, seed: int) -> np.ndarray:
    bits = np.zeros(R * R * (R // 64), np.uint64)
    check(lib().vx_synth_urban(R, hmin, hmax, seed, _p(bits)))
    return bits


def synth_rgba8(brick_coord: np.ndarray, seed: int) -> np.ndarray:
    bc = np.ascontiguousarray(brick_coord, np.uint32)
    out = np.zeros(bc.size * 512, np.uint32)
    check(lib().vx_synth_rgba8(_p(bc), bc.size, seed, _p(out)))
    return out


def synth_dxt1(brick_coord: np.ndarray, seed: int) -> np.ndarray:
    bc = np.ascontiguousarray(brick_coord, np.uint32)
    out = np.zeros(bc.size * 32, np.uint64)
    check(lib().vx_synth_dxt1(_p(bc), bc.size, seed, _p(out)))
    return out


@dataclass
class SceneArrays:
    """Host copy of a scene in the device layout of vx.h."""
    world_min: tuple
    world_max: tuple
    max_levels: int
    bricks_per_axis: int
    nodes: np.ndarray        # u32 pairs {child_ptr, valid | leaf << 8}
    node_brick: np.ndarray
    grid_lookup: np.ndarray
    brick_coord: np.ndarray
    brick_occ: np.ndarray    # 16 u32 per brick
    color_kind: int = VX_COLOR_NONE
    brick_color: np.ndarray | None = None
    brick_normal: np.ndarray | None = None  # (bricks, 32, 2) u64 DXT normal blocks (build_normals)

    @property
    def node_count(self) -> int:
        return self.nodes.size // 2

    @property
    def brick_count(self) -> int:
        return self.brick_coord.size


def build_dense(bits: np.ndarray, R: int, max_levels: int) -> SceneArrays:
    """LaineKarrasOctree::rebuild + VoxelSceneCacher packing for a dense grid
    with world bounds [0,R]^3 (vx_build_dense)."""
    bits = np.ascontiguousarray(bits, np.uint64)
    assert bits.size == R * R * (R // 64)
    h = C.c_void_p()
    check(lib().vx_build_dense(_p(bits), R, max_levels, C.byref(h)))
    try:
        d = _SceneDesc()
        check(lib().vx_build_desc(h, C.byref(d)))
        bpa = d.config.bricks_per_axis

        def take(ptr, n, dt):
            if n == 0 or not ptr:
                return np.zeros(0, dt)
            buf = (C.c_char * (n * np.dtype(dt).itemsize)).from_address(ptr)
            return np.frombuffer(buf, dtype=dt, count=n).copy()

        return SceneArrays(tuple(d.config.world_min), tuple(d.config.world_max), d.config.max_levels, bpa,
                           take(d.nodes, 2 * d.node_count, np.uint32), take(d.node_brick, d.node_count, np.uint32),
                           take(d.grid_lookup, bpa ** 3, np.uint32), take(d.brick_coord, d.brick_count, np.uint32),
                           take(d.brick_occ, 16 * d.brick_count, np.uint32))
    finally:
        lib().vx_build_free(h)


def bounds_checks():
    """vx_bounds_checks: (checked build loaded, violation bits since the last call)."""
    en, v = C.c_int32(), C.c_uint32()
    check(lib().vx_bounds_checks(C.byref(en), C.byref(v)))
    return bool(en.value), v.value


def build_normals(brick_occ: np.ndarray) -> np.ndarray:
    """DXT normal payload (bricks, 32, 2) u64 from 16-word brick occupancy (vx_build_normals, host)."""
    occ = np.ascontiguousarray(brick_occ, np.uint32).reshape(-1, 16)
    out = np.zeros((occ.shape[0], 32, 2), np.uint64)
    check(lib().vx_build_normals(_p(occ), occ.shape[0], _p(out)))
    return out


def build_dxt1(rgb: np.ndarray, brick_occ: np.ndarray) -> np.ndarray:
    """DXT1 colour payload (bricks*32 u64) from per-voxel RGB floats (bricks, 512, 3) (vx_build_dxt1, host)."""
    occ = np.ascontiguousarray(brick_occ, np.uint32).reshape(-1, 16)
    c = np.ascontiguousarray(rgb, np.float32).reshape(occ.shape[0], 512, 3)
    out = np.zeros(occ.shape[0] * 32, np.uint64)
    check(lib().vx_build_dxt1(_p(c), _p(occ), occ.shape[0], _p(out)))
    return out


def material_rgb(words: np.ndarray) -> np.ndarray:
    """vx_material_rgb: MaterialIdToColor of every material word, (n, 3) float32 (host)."""
    w = np.ascontiguousarray(words, np.uint32).reshape(-1)
    out = np.zeros((w.size, 3), np.float32)
    check(lib().vx_material_rgb(_p(w), w.size, _p(out)))
    return out


def material_rgb_dev(words, out, stream=None):
    """vx_material_rgb_dev: words (n) 32-bit CUDA tensor -> out (n*3) float32 CUDA tensor."""
    check(lib().vx_material_rgb_dev(_p(words), words.numel(), _p(out), _stream(stream)))


def build_dxt1_dev(rgb, occ, out, stream=None):
    """vx_build_dxt1_dev: rgb (bricks*512*3) float32, occ (bricks*16) 32-bit, out (bricks*32) 8-byte CUDA tensors."""
    check(lib().vx_build_dxt1_dev(_p(rgb), _p(occ), occ.numel() // 16, _p(out), _stream(stream)))


def build_normals_dev(occ, out, stream=None):
    """vx_build_normals_dev: occ (bricks*16) u32/int32 CUDA tensor -> out (bricks*64) 8-byte CUDA tensor."""
    check(lib().vx_build_normals_dev(_p(occ), occ.numel() // 16, _p(out), _stream(stream)))


def scene_from_dense_dev(bits, R: int, max_levels: int, color_kind: int = VX_COLOR_NONE, color_seed: int = 0,
                         with_normals: bool = False, stream=None) -> "Scene":
    """vx_scene_create_dense_dev: bits is an (R^3/64) 8-byte CUDA tensor (vx_synth_noise_dev's output)."""
    h = C.c_void_p()
    check(lib().vx_scene_create_dense_dev(_p(bits), R, max_levels, color_kind, color_seed, int(with_normals),
                                          C.byref(h), _stream(stream)))
    return Scene.from_handle(h)


def nodes_from_reference(ref_nodes: np.ndarray):
    ref = np.ascontiguousarray(ref_nodes, np.uint64)
    nodes = np.zeros(2 * ref.size, np.uint32)
    nb = np.zeros(ref.size, np.uint32)
    check(lib().vx_nodes_from_reference(_p(ref), ref.size, _p(nodes), _p(nb)))
    return nodes, nb


def camera_rays(pc: CameraPC, width: int, height: int) -> np.ndarray:
    """Primary rays exactly as vx_render generates them (N x 6 float32)."""
    out = np.zeros((width * height, 6), np.float32)
    check(lib().vx_camera_rays(C.byref(pc), width, height, _p(out)))
    return out


# ---------------------------------------------------------------------------
# Device scene
# ---------------------------------------------------------------------------

def _desc_of(a: SceneArrays):
    """vx_scene_desc pointing into the host arrays of `a` (kept alive by the returned list)."""
    d = _SceneDesc()
    d.config.world_min[:] = [float(v) for v in a.world_min]
    d.config.world_max[:] = [float(v) for v in a.world_max]
    d.config.max_levels = a.max_levels
    d.config.brick_depth = 3
    d.config.bricks_per_axis = a.bricks_per_axis
    keep = [np.ascontiguousarray(x, np.uint32) for x in (a.nodes, a.node_brick, a.grid_lookup, a.brick_coord,
                                                         a.brick_occ)]
    d.nodes, d.node_brick, d.grid_lookup, d.brick_coord, d.brick_occ = [_p(x) for x in keep]
    d.node_count = a.node_count
    d.brick_count = a.brick_count
    d.color_kind = a.color_kind
    if a.brick_color is not None:
        keep.append(np.ascontiguousarray(a.brick_color))
        d.brick_color = _p(keep[-1])
    if a.brick_normal is not None:
        assert a.brick_normal.size == a.brick_count * 64
        keep.append(np.ascontiguousarray(a.brick_normal, np.uint64))
        d.brick_normal = _p(keep[-1])
    return d, keep


def _arrays_of_cache(h, materials=False) -> SceneArrays:
    d = _SceneDesc()
    check((lib().vx_cache_desc_materials if materials else lib().vx_cache_desc)(h, C.byref(d)))
    bpa, B, D = d.config.bricks_per_axis, d.brick_count, d.node_count

    def take(ptr, n, dt):
        if n == 0 or not ptr:
            return np.zeros(0, dt)
        buf = (C.c_char * (n * np.dtype(dt).itemsize)).from_address(ptr)
        return np.frombuffer(buf, dtype=dt, count=n).copy()

    color = None
    if d.color_kind in (VX_COLOR_RGBA8, VX_COLOR_MATERIAL):
        color = take(d.brick_color, 512 * B, np.uint32)
    elif d.color_kind == VX_COLOR_DXT1:
        color = take(d.brick_color, 32 * B, np.uint64)
    normal = take(d.brick_normal, 64 * B, np.uint64).reshape(B, 32, 2) if d.brick_normal else None
    return SceneArrays(tuple(d.config.world_min), tuple(d.config.world_max), d.config.max_levels, bpa,
                       take(d.nodes, 2 * D, np.uint32), take(d.node_brick, D, np.uint32),
                       take(d.grid_lookup, bpa ** 3, np.uint32), take(d.brick_coord, B, np.uint32),
                       take(d.brick_occ, 16 * B, np.uint32), d.color_kind if color is not None else VX_COLOR_NONE,
                       color, normal)


def cache_write(path: str, arrays: SceneArrays):
    """vx_cache_write (VXSC)."""
    d, keep = _desc_of(arrays)
    check(lib().vx_cache_write(os.fsencode(path), C.byref(d)))


def cache_read(path: str) -> SceneArrays:
    """vx_cache_read (VXSC) -> host arrays."""
    h = C.c_void_p()
    check(lib().vx_cache_read(os.fsencode(path), C.byref(h)))
    try:
        return _arrays_of_cache(h)
    finally:
        lib().vx_cache_free(h)


def cache_write_vsca(path: str, arrays: SceneArrays, scene_type: int, resolution: int, density: float, seed: int):
    """vx_cache_write_vsca: the reference's VoxelSceneCacher file format."""
    d, keep = _desc_of(arrays)
    check(lib().vx_cache_write_vsca(os.fsencode(path), C.byref(d), scene_type, resolution, float(density), seed))


def cache_read_vsca(path: str, entry: int = 0, materials: bool = False) -> SceneArrays:
    """vx_cache_read_vsca -> host arrays; colour = the file's DXT1 colours (vx_cache_desc), or its
    brickData material words with materials=True (vx_cache_desc_materials)."""
    h = C.c_void_p()
    check(lib().vx_cache_read_vsca(os.fsencode(path), entry, C.byref(h)))
    try:
        return _arrays_of_cache(h, materials)
    finally:
        lib().vx_cache_free(h)


class _SceneInfo(C.Structure):
    _fields_ = [("config", _Config), ("node_count", C.c_uint32), ("brick_count", C.c_uint32),
                ("color_kind", C.c_int32), ("has_normals", C.c_int32)]


class Scene:
    """A scene resident in device memory (vx_scene)."""

    @classmethod
    def from_handle(cls, handle: C.c_void_p) -> "Scene":
        """Wraps a vx_scene made by the library (vx_scene_create_dense_dev); the
        host arrays are downloaded on first use of .arrays."""
        self = cls.__new__(cls)
        self._h = handle
        self._arrays = None
        return self

    def info(self):
        i = _SceneInfo()
        check(lib().vx_scene_info_get(self._h, C.byref(i)))
        return i

    @property
    def arrays(self) -> SceneArrays:
        if self._arrays is None:
            self._arrays = self.download()
        return self._arrays

    def download(self) -> SceneArrays:
        """vx_scene_download: every device array back in host memory."""
        i = self.info()
        bpa, B, D = i.config.bricks_per_axis, i.brick_count, i.node_count
        nodes, nb = np.zeros(2 * D, np.uint32), np.zeros(D, np.uint32)
        grid, coord, occ = np.zeros(bpa ** 3, np.uint32), np.zeros(B, np.uint32), np.zeros(16 * B, np.uint32)
        color = None
        if i.color_kind in (VX_COLOR_RGBA8, VX_COLOR_MATERIAL):
            color = np.zeros(512 * B, np.uint32)
        elif i.color_kind == VX_COLOR_DXT1:
            color = np.zeros(32 * B, np.uint64)
        normal = np.zeros((B, 32, 2), np.uint64) if i.has_normals else None
        check(lib().vx_scene_download(self._h, _p(nodes), _p(nb), _p(grid), _p(coord), _p(occ), _p(color),
                                      _p(normal)))
        return SceneArrays(tuple(i.config.world_min), tuple(i.config.world_max), i.config.max_levels, bpa, nodes,
                           nb, grid, coord, occ, i.color_kind, color, normal)

    def __init__(self, arrays: SceneArrays):
        self._arrays = arrays
        d, keep = _desc_of(arrays)
        self._h = C.c_void_p()
        check(lib().vx_scene_create(C.byref(d), C.byref(self._h)))
        del keep  # the scene holds device copies

    @classmethod
    def load(cls, path: str) -> "Scene":
        """vx_scene_load: a VXSC cache file straight into a device scene."""
        h = C.c_void_p()
        check(lib().vx_scene_load(os.fsencode(path), C.byref(h)))
        return cls.from_handle(h)

    def save(self, path: str):
        """vx_scene_save: the scene's arrays into a VXSC cache file."""
        check(lib().vx_scene_save(self._h, os.fsencode(path)))

    @property
    def handle(self):
        return self._h

    @property
    def color_kind(self) -> int:
        return self._arrays.color_kind if self._arrays is not None else self.info().color_kind

    def device_bytes(self) -> int:
        v = C.c_uint64()
        check(lib().vx_scene_device_bytes(self._h, C.byref(v)))
        return v.value

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            check(lib().vx_scene_destroy(self._h))
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- device-buffer calls (torch tensors) --------------------------------
    def color_width(self) -> int:
        return {VX_COLOR_NONE: 0, VX_COLOR_RGBA8: 1, VX_COLOR_DXT1: 3, VX_COLOR_MATERIAL: 1}[self.color_kind]

    def cast_rays_dev(self, rays, hits, color=None, counters=None, t_min=0.0, t_max=FLT_MAX, stream=None, lod=None):
        """rays: (n,6) float32 CUDA tensor; hits: (n,4) int32/uint32 CUDA tensor (16 B per ray).
        lod: LodParams for castRayWithLOD (vx_cast_rays_lod), None for castRay."""
        import torch
        n = rays.shape[0]
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        if lod is None:
            check(lib().vx_cast_rays(self._h, _p(rays), n, float(t_min), float(t_max), _p(hits), _p(color),
                                     _p(counters), C.c_void_p(s)))
        else:
            check(lib().vx_cast_rays_lod(self._h, _p(rays), n, float(t_min), float(t_max), C.byref(_lod(lod)),
                                         _p(hits), _p(color), _p(counters), C.c_void_p(s)))

    def cast_shadow_rays_dev(self, rays, hits, light_dir, shadow_hits, t_min=0.0, t_max=FLT_MAX, stream=None):
        """vx_cast_shadow_rays: the shadow ray of every primary hit, compacted and cast; shadow_hits
        (n,4) gets what spawn_shadow_rays + cast_rays_dev over all n slots would write."""
        ld = (C.c_float * 3)(*[float(v) for v in light_dir])
        check(lib().vx_cast_shadow_rays(self._h, _p(rays), _p(hits), rays.shape[0], ld, float(t_min), float(t_max),
                                        _p(shadow_hits), _stream(stream)))

    def hit_normals_dev(self, hits, out, stream=None):
        """vx_hit_normals: hits (n,4) CUDA tensor -> out (n,3) float32 CUDA tensor."""
        check(lib().vx_hit_normals(self._h, _p(hits), hits.shape[0], _p(out), _stream(stream)))

    def render_dev(self, pc: CameraPC, width: int, height: int, image=None, hits=None, color=None, stream=None):
        import torch
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        check(lib().vx_render(self._h, C.byref(pc), width, height, _p(image), _p(hits), _p(color), C.c_void_p(s)))

    # -- host-buffer calls ---------------------------------------------------
    def cast_rays_host(self, rays: np.ndarray, t_min=0.0, t_max=FLT_MAX, with_color=True, lod=None):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        hits = np.zeros(rays.shape[0], HIT_DTYPE)
        cw = self.color_width()
        color = None
        if with_color and cw:
            color = np.zeros((rays.shape[0], cw), np.uint32 if cw == 1 else np.float32)
        if lod is None:
            check(lib().vx_cast_rays_host(self._h, _p(rays), rays.shape[0], float(t_min), float(t_max), _p(hits),
                                          _p(color), None))
        else:
            check(lib().vx_cast_rays_host_lod(self._h, _p(rays), rays.shape[0], float(t_min), float(t_max),
                                              C.byref(_lod(lod)), _p(hits), _p(color), None))
        return hits, color


class LodParams(C.Structure):
    """LODParameters (SVO/include/SVOLOD.h:50-177): vx_lod_params."""
    _fields_ = [("ray_orig_size", C.c_float), ("ray_dir_size", C.c_float)]

    def as_tuple(self):
        return (self.ray_orig_size, self.ray_dir_size)


def _lod(lod) -> LodParams:
    return lod if isinstance(lod, LodParams) else LodParams(float(lod[0]), float(lod[1]))


def lod_from_camera(fov_y: float, screen_height: int, near_plane: float = 0.0) -> LodParams:
    """LODParameters::fromCamera (near_plane 0) / fromCameraWithNearPlane."""
    out = LodParams()
    check(lib().vx_lod_from_camera(float(fov_y), int(screen_height), float(near_plane), C.byref(out)))
    return out


def lod_with_bias(lod, bias: float) -> LodParams:
    """LODParameters::withBias: both sizes times 2^bias."""
    out = LodParams()
    check(lib().vx_lod_with_bias(C.byref(_lod(lod)), float(bias), C.byref(out)))
    return out


# ---------------------------------------------------------------------------
# ISVOStructure-shaped facade
# ---------------------------------------------------------------------------

@dataclass
class RayHit:
    """ISVOStructure::RayHit (SVO/include/ISVOStructure.h:101-112)."""
    hit: bool
    tMin: float
    tMax: float
    hitPoint: tuple
    normal: tuple
    scale: int
    brick: int
    voxel: int
    node: int
    entity: tuple | None  # integer voxel position of the hit (the entity's MortonKey position)


class CudaOctree:
    """Drop-in for LaineKarrasOctree::castRay on a device-resident scene."""

    def __init__(self, scene: Scene):
        self.scene = scene
        a = scene.arrays
        self.world_min = np.array(a.world_min, np.float32)
        self.max_levels = a.max_levels

    def castRays(self, origins, directions, tMin=0.0, tMax=FLT_MAX, lod=None):
        o = np.asarray(origins, np.float32).reshape(-1, 3)
        d = np.asarray(directions, np.float32).reshape(-1, 3)
        hits, _ = self.scene.cast_rays_host(np.concatenate([o, d], axis=1), tMin, tMax, with_color=False, lod=lod)
        return hits

    def castRayWithLOD(self, origin, direction, lod, tMin=0.0, tMax=FLT_MAX) -> RayHit:
        """LaineKarrasOctree::castRayWithLOD (SVOTraversal.cpp:224-232)."""
        return self.castRay(origin, direction, tMin, tMax, lod=lod)

    def castRayLOD(self, origin, direction, lodBias, tMin=0.0, tMax=FLT_MAX) -> RayHit:
        """castRayLOD (SVOTraversal.cpp:198-209): the bias is the cone spread, origin size 0."""
        return self.castRay(origin, direction, tMin, tMax, lod=LodParams(0.0, float(lodBias)))

    def castRayScreenSpaceLOD(self, origin, direction, fovY, screenHeight, tMin=0.0, tMax=FLT_MAX) -> RayHit:
        """castRayScreenSpaceLOD (SVOTraversal.cpp:211-222)."""
        return self.castRay(origin, direction, tMin, tMax, lod=lod_from_camera(fovY, screenHeight))

    def castRay(self, origin, direction, tMin=0.0, tMax=FLT_MAX, lod=None) -> RayHit:
        h = self.castRays([origin], [direction], tMin, tMax, lod=lod)[0]
        if not (h["flags"] & VX_HIT_HIT):
            return RayHit(False, 0.0, 0.0, (0.0, 0.0, 0.0), (0.0, 0.0, 0.0), 0, NONE, 0xFFFF, NONE, None)
        o = np.asarray(origin, np.float32)
        d = np.asarray(direction, np.float32)
        dn = d * (np.float32(1.0) / np.sqrt((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]))
        t = np.float32(h["t"])
        hp = tuple(float(v) for v in (o + dn * t))
        if h["brick"] == NONE:
            # LOD hit (SVOTraversal.cpp:639-649): tMax = t + the cell's world size
            # 2^(user scale - max_levels) * worldSize.x, normal +y, no entity.
            wsx = np.float32(self.scene.arrays.world_max[0]) - np.float32(self.scene.arrays.world_min[0])
            size = np.float32(np.ldexp(np.float32(1.0), int(h["scale"]) - self.max_levels)) * wsx
            return RayHit(True, float(t), float(t + size), hp, (0.0, 1.0, 0.0), int(h["scale"]), NONE, 0xFFFF,
                          int(h["node"]), None)
        axis = (int(h["flags"]) >> 1) & 3
        n = [0.0, 0.0, 0.0]
        n[axis] = -1.0 if h["flags"] & VX_HIT_NORMAL_NEG else 1.0
        bc = int(self.scene.arrays.brick_coord[h["brick"]])
        v = int(h["voxel"])
        q = np.floor(self.world_min).astype(np.int64)
        ent = ((bc & 0x3FF) * 8 + (v & 7) + int(q[0]), ((bc >> 10) & 0x3FF) * 8 + ((v >> 3) & 7) + int(q[1]),
               ((bc >> 20) & 0x3FF) * 8 + (v >> 6) + int(q[2]))
        return RayHit(True, float(t), float(t + np.float32(1.0)), hp, tuple(n), int(h["scale"]),
                      int(h["brick"]), v, int(h["node"]), ent)


# ---------------------------------------------------------------------------
# Batched form
# ---------------------------------------------------------------------------

class BatchTuning(C.Structure):
    _fields_ = [("block", C.c_int32), ("rays_per_task", C.c_int32), ("stack_in_shared", C.c_int32),
                ("refill", C.c_int32), ("budget", C.c_int32)]

    def as_dict(self):
        return {"block": self.block, "rays_per_task": self.rays_per_task, "stack_in_shared": self.stack_in_shared,
                "refill": self.refill, "budget": self.budget}


def _stream(stream):
    import torch
    return C.c_void_p(stream if stream is not None else torch.cuda.current_stream().cuda_stream)


class Batch:
    """Scenes cast together by the persistent batched kernel (vx_batch)."""

    def __init__(self, scenes):
        self.scenes = list(scenes)
        arr = (C.c_void_p * len(self.scenes))(*[sc.handle.value for sc in self.scenes])
        self._h = C.c_void_p()
        check(lib().vx_batch_create(arr, len(self.scenes), C.byref(self._h)))

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            check(lib().vx_batch_destroy(self._h))
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def tuning(self) -> BatchTuning:
        t = BatchTuning()
        check(lib().vx_batch_get_tuning(self._h, C.byref(t)))
        return t

    def set_tuning(self, block=256, rays_per_task=32, stack_in_shared=1, refill=0, budget=0):
        t = BatchTuning(block, rays_per_task, stack_in_shared, refill, budget)
        check(lib().vx_batch_set_tuning(self._h, C.byref(t)))

    def set_bounce_tuning(self, tuning=None):
        """Tuning of the bounce pass of frames captured later (None: the batch's own)."""
        check(lib().vx_batch_set_bounce_tuning(self._h, None if tuning is None else C.byref(tuning)))

    def cast(self, rays, begin, hits, counters=None, t_min=0.0, t_max=FLT_MAX, stream=None):
        check(lib().vx_cast_batch(self._h, _p(rays), _p(begin), rays.shape[0], float(t_min), float(t_max), _p(hits),
                                  _p(counters), _stream(stream)))

    def autotune(self, rays, begin, hits, stream=None):
        t = BatchTuning()
        ms = C.c_float()
        check(lib().vx_batch_autotune(self._h, _p(rays), _p(begin), rays.shape[0], _p(hits), _stream(stream),
                                      C.byref(t), C.byref(ms)))
        return t, ms.value

    def capture_frame(self, primary, primary_begin, primary_hits, bounce, bounce_begin, bounce_hits, seed, stream):
        check(lib().vx_batch_capture_frame(self._h, _p(primary), _p(primary_begin), primary.shape[0],
                                           _p(primary_hits), _p(bounce), _p(bounce_begin), _p(bounce_hits), seed,
                                           C.c_void_p(stream)))

    def capture_frame_compact(self, primary, primary_begin, primary_hits, bounce, bounce_hits, seed, stream):
        """vx_batch_capture_frame_compact: the bounce pass casts only the bounce rays of primary hits
        (compacted into `bounce`, 2 * hits of its 2n rows, per scene grouped by direction bin);
        `bounce_hits` ends up as with capture_frame."""
        check(lib().vx_batch_capture_frame_compact(self._h, _p(primary), _p(primary_begin), primary.shape[0],
                                                   _p(primary_hits), _p(bounce), _p(bounce_hits), seed,
                                                   C.c_void_p(stream)))

    def capture_frame_parts(self, primary, primary_begin, primary_hits, bounce, bounce_hits, seed, parts, stream):
        """vx_batch_capture_frame_parts: the compacted frame as `parts` pieces of consecutive primary
        rays, each with its own graph; launch_frame_host overlaps each piece's copies with the casts
        of the others.  Results as with capture_frame_compact."""
        check(lib().vx_batch_capture_frame_parts(self._h, _p(primary), _p(primary_begin), primary.shape[0],
                                                 _p(primary_hits), _p(bounce), _p(bounce_hits), seed, int(parts),
                                                 C.c_void_p(stream)))

    def launch_frame(self, stream=None):
        check(lib().vx_batch_launch_frame(self._h, _stream(stream)))

    def launch_frame_host(self, primary_host, primary_hits_host, bounce_hits_host, stream=None):
        """vx_batch_launch_frame_host: the captured frame from host buffers (rays in, both hit
        buffers out); returns when the results are in host memory."""
        check(lib().vx_batch_launch_frame_host(self._h, _p(primary_host), _p(primary_hits_host),
                                               _p(bounce_hits_host), _stream(stream)))

    def frame_compaction(self):
        """vx_batch_frame_compaction after a compacted frame has run: (scene offsets of the
        compacted bounce rays, count + 1 entries; hit slot of every compacted ray)."""
        sb = np.zeros(len(self.scenes) + 1, np.uint32)
        check(lib().vx_batch_frame_compaction(self._h, _p(sb), None, None, None))
        mp = np.zeros(int(sb[-1]), np.uint32)
        check(lib().vx_batch_frame_compaction(self._h, None, _p(mp), None, None))
        return sb, mp


def spawn_bounce_rays(rays, hits, seed, out, stream=None):
    check(lib().vx_spawn_bounce_rays(_p(rays), _p(hits), rays.shape[0], seed, _p(out), _stream(stream)))


def spawn_shadow_rays(rays, hits, light_dir, out, stream=None):
    ld = (C.c_float * 3)(*[float(v) for v in light_dir])
    check(lib().vx_spawn_shadow_rays(_p(rays), _p(hits), rays.shape[0], ld, _p(out), _stream(stream)))


def bounce_table() -> np.ndarray:
    out = np.zeros(4096 * 3, np.float32)
    check(lib().vx_bounce_table(_p(out)))
    return out.reshape(4096, 3)


VX_NOALLOC_MAX_SCENES = 64


def cast_batch_noalloc(scenes, rays, begin, hits, t_min=0.0, t_max=FLT_MAX, stream=None):
    """vx_cast_batch_noalloc: the batched cast without any device allocation, for
    callers that cannot allocate device memory (a fixed device-memory budget owned by
    the host application, or a frame loop that cannot take cudaMalloc's implicit
    synchronisation).  At most VX_NOALLOC_MAX_SCENES scenes; calls must not overlap
    on the GPU (they share one static scratch array)."""
    arr = (C.c_void_p * len(scenes))(*[sc.handle.value for sc in scenes])
    check(lib().vx_cast_batch_noalloc(arr, len(scenes), _p(rays), _p(begin), rays.shape[0], float(t_min),
                                      float(t_max), _p(hits), _stream(stream)))


# ---------------------------------------------------------------------------
# Differentiable form
# ---------------------------------------------------------------------------
VX_DIFF_VOXEL_RGB, VX_DIFF_DXT1_ENDPOINTS = 0, 1


def diff_forward(scene: "Scene", pc: CameraPC, width: int, height: int, kind: int, attr, dxt_idx, image, record,
                 stream=None):
    check(lib().vx_diff_forward(scene.handle, C.byref(pc), width, height, kind, _p(attr), _p(dxt_idx), _p(image),
                                _p(record), _stream(stream)))


def diff_forward_views(scene: "Scene", pcs, width: int, height: int, kind: int, attr, dxt_idx, image, record,
                       stream=None):
    """vx_diff_forward_views: all cameras in one launch; image (views*w*h, 3), record (views*w*h, 4)."""
    arr = (CameraPC * len(pcs))(*pcs)
    check(lib().vx_diff_forward_views(scene.handle, arr, len(pcs), width, height, kind, _p(attr), _p(dxt_idx),
                                      _p(image), _p(record), _stream(stream)))


def diff_backward(kind: int, dxt_idx, record, image, target, grad, loss=None, stream=None):
    check(lib().vx_diff_backward(record.shape[0], kind, _p(dxt_idx), _p(record), _p(image), _p(target), _p(grad),
                                 _p(loss), _stream(stream)))
