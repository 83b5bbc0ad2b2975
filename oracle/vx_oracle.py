"""ctypes binding of the CPU oracle (oracle/libvx_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and the CPU
baseline leg of bench.py.  The product (libvx.so and its Python binding)
never imports this module.  See vx_oracle.h for what the oracle restates and
for its parity status.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libvx_oracle.so")

HIT_DTYPE = np.dtype([
    ("t", "<f4"), ("t_exit", "<f4"), ("hit_point", "<f4", 3), ("normal", "<f4", 3),
    ("brick", "<u4"), ("node", "<u4"), ("voxel", "<u4"), ("key", "<i4", 3),
    ("scale", "<i4"), ("flags", "<u4"), ("iters", "<u4"), ("grid_reads", "<u4"),
    ("dda_steps", "<u4"), ("leaf_visits", "<u4"),
])

_lib = None


def build() -> None:
    """Compile the oracle with its Makefile (plain g++)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp, u32, u64, i32, f32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int32, C.c_float
        L.vxo_build_from_keys.restype = vp
        L.vxo_build_from_keys.argtypes = [vp, u64, vp, vp, C.c_int, C.c_int, C.c_char_p, C.c_int]
        L.vxo_build_from_dense.restype = vp
        L.vxo_build_from_dense.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_int]
        L.vxo_build_from_descriptors.restype = vp
        L.vxo_build_from_descriptors.argtypes = [vp, vp, u32, vp, vp, C.c_int, C.c_int]
        L.vxo_free.argtypes = [vp]
        for f in ("vxo_node_count", "vxo_brick_count", "vxo_max_child_pointer"):
            getattr(L, f).restype = u32
            getattr(L, f).argtypes = [vp]
        L.vxo_bricks_per_axis.restype = i32
        L.vxo_bricks_per_axis.argtypes = [vp]
        L.vxo_export.argtypes = [vp, vp, vp, vp, vp, vp]
        L.vxo_cast_rays.argtypes = [vp, vp, u64, f32, f32, vp, C.c_int]
        L.vxo_cast_rays_lod.argtypes = [vp, vp, u64, f32, f32, f32, f32, vp, C.c_int]
        L.vxo_lod_from_camera.argtypes = [f32, i32, f32, vp]
        L.vxo_lod_with_bias.argtypes = [vp, f32, vp]
        L.vxo_dxt1_decode_head.argtypes = [u32, vp]
        L.vxo_dxt1_decode_block.argtypes = [u64, vp]
        L.vxo_dxt1_encode_head.restype = u32
        L.vxo_dxt1_encode_head.argtypes = [vp, vp]
        L.vxo_dxt1_encode_block.restype = u64
        L.vxo_dxt1_encode_block.argtypes = [vp, u64, vp]
        L.vxo_hit_texel_dxt.argtypes = [vp, u32, u32, vp]
        L.vxo_camera_rays.argtypes = [vp, u32, u32, vp, vp]
        L.vxo_synth_noise.restype = C.c_int
        L.vxo_synth_noise.argtypes = [u32, u32, u32, f32, u64, i32, vp, C.c_int]
        L.vxo_synth_urban.restype = C.c_int
        L.vxo_synth_urban.argtypes = [u32, u32, u32, u64, vp]
        L.vxo_bounce_table.argtypes = [vp]
        L.vxo_material_color_cpu.argtypes = [u32, vp]
        L.vxo_material_color_shader.argtypes = [u32, vp]
        L.vxo_spawn_rays.argtypes = [vp, vp, vp, u64, C.c_int, u64, vp, vp]
        L.vxo_hit_texels_dxt.argtypes = [vp, u64, vp, vp, vp]
        L.vxo_shade.restype = u32
        L.vxo_shade.argtypes = [vp, C.c_int, C.c_int, C.c_int, f32]
        L.vxo_dxtn_encode_block.argtypes = [vp, u64, vp, vp]
        L.vxo_dxtn_decode_block.argtypes = [vp, vp]
        L.vxo_encode_raw_normal.restype = u32
        L.vxo_encode_raw_normal.argtypes = [vp]
        L.vxo_geometric_normals.argtypes = [vp, vp]
        L.vxo_brick_normals.argtypes = [vp, u64, vp, C.c_int]
        L.vxo_hit_normal_dxt.argtypes = [vp, u32, u32, vp]
        L.vxo_brick_dxt1.argtypes = [vp, vp, u64, vp]
        L.vxo_shade_dxt_normal.restype = u32
        L.vxo_shade_dxt_normal.argtypes = [vp, C.c_int, vp, C.c_int, C.c_int, f32]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class OracleScene:
    """Octree built by the restated LaineKarrasOctree::rebuild."""

    def __init__(self, handle):
        self._h = handle
        L = lib()
        self.node_count = L.vxo_node_count(handle)
        self.brick_count = L.vxo_brick_count(handle)
        self.bricks_per_axis = L.vxo_bricks_per_axis(handle)
        self.max_child_pointer = L.vxo_max_child_pointer(handle)

    @classmethod
    def from_keys(cls, keys, world_min, world_max, max_levels, brick_depth=3):
        keys = np.ascontiguousarray(np.asarray(keys, dtype=np.int32).reshape(-1, 3))
        wmin = np.asarray(world_min, dtype=np.float32)
        wmax = np.asarray(world_max, dtype=np.float32)
        err = C.create_string_buffer(256)
        h = lib().vxo_build_from_keys(_ptr(keys), keys.shape[0], _ptr(wmin), _ptr(wmax),
                                      max_levels, brick_depth, err, 256)
        if not h:
            raise ValueError(err.value.decode())
        return cls(h)

    @classmethod
    def from_positions(cls, positions, world_min, world_max, max_levels, brick_depth=3):
        """Voxels given as float world positions, quantised the way
        MortonCode64::fromWorldPos(float) does (floor(p + 1e-5),
        Core/src/MortonEncoding.cpp:99-108)."""
        p = np.asarray(positions, dtype=np.float32).reshape(-1, 3)
        keys = np.floor(p + np.float32(1e-5)).astype(np.int32)
        return cls.from_keys(keys, world_min, world_max, max_levels, brick_depth)

    @classmethod
    def from_dense(cls, bits: np.ndarray, R: int, max_levels: int, brick_depth: int = 3):
        bits = np.ascontiguousarray(bits, dtype=np.uint64)
        assert bits.size == R * R * (R // 64)
        err = C.create_string_buffer(256)
        h = lib().vxo_build_from_dense(_ptr(bits), R, max_levels, brick_depth, err, 256)
        if not h:
            raise ValueError(err.value.decode())
        return cls(h)

    @classmethod
    def from_descriptors(cls, nodes, node_brick, world_min, world_max, max_levels, brick_depth=3):
        nodes = np.ascontiguousarray(nodes, dtype=np.uint32).reshape(-1)
        nb = None if node_brick is None else np.ascontiguousarray(node_brick, dtype=np.uint32)
        wmin = np.asarray(world_min, dtype=np.float32)
        wmax = np.asarray(world_max, dtype=np.float32)
        h = lib().vxo_build_from_descriptors(_ptr(nodes), _ptr(nb), nodes.size // 2, _ptr(wmin),
                                             _ptr(wmax), max_levels, brick_depth)
        return cls(h)

    def export(self):
        """Octree in the product's device layout (see vx.h)."""
        D, B, bpa = self.node_count, self.brick_count, self.bricks_per_axis
        nodes = np.zeros(2 * D, np.uint32)
        node_brick = np.zeros(D, np.uint32)
        grid = np.zeros(bpa ** 3, np.uint32)
        coord = np.zeros(B, np.uint32)
        occ = np.zeros(16 * B, np.uint32)
        lib().vxo_export(self._h, _ptr(nodes), _ptr(node_brick), _ptr(grid), _ptr(coord), _ptr(occ))
        return dict(nodes=nodes, node_brick=node_brick, grid_lookup=grid, brick_coord=coord,
                    brick_occ=occ)

    def cast_rays(self, rays: np.ndarray, t_min=0.0, t_max=3.4028234663852886e38, threads=0):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
        out = np.zeros(rays.shape[0], HIT_DTYPE)
        lib().vxo_cast_rays(self._h, _ptr(rays), rays.shape[0], float(t_min), float(t_max),
                            _ptr(out), int(threads))
        return out

    def cast_rays_lod(self, rays: np.ndarray, lod, t_min=0.0, t_max=3.4028234663852886e38, threads=0):
        """castRayWithLOD over many rays; lod = (rayOrigSize, rayDirSize)."""
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
        out = np.zeros(rays.shape[0], HIT_DTYPE)
        lib().vxo_cast_rays_lod(self._h, _ptr(rays), rays.shape[0], float(t_min), float(t_max), float(lod[0]),
                                float(lod[1]), _ptr(out), int(threads))
        return out

    def castRay(self, origin, direction, tMin=0.0, tMax=3.4028234663852886e38):
        r = np.array([list(origin) + list(direction)], np.float32)
        return self.cast_rays(r, tMin, tMax, threads=1)[0]

    def castRayWithLOD(self, origin, direction, lod, tMin=0.0, tMax=3.4028234663852886e38):
        r = np.array([list(origin) + list(direction)], np.float32)
        return self.cast_rays_lod(r, lod, tMin, tMax, threads=1)[0]

    def castRayLOD(self, origin, direction, lodBias, tMin=0.0, tMax=3.4028234663852886e38):
        """SVOTraversal.cpp:198-209: the bias is the cone spread itself."""
        return self.castRayWithLOD(origin, direction, (0.0, lodBias), tMin, tMax)

    def castRayScreenSpaceLOD(self, origin, direction, fovY, screenHeight, tMin=0.0, tMax=3.4028234663852886e38):
        return self.castRayWithLOD(origin, direction, lod_from_camera(fovY, screenHeight), tMin, tMax)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().vxo_free(self._h)
            self._h = None


def lod_from_camera(fov_y: float, screen_height: int, near_plane: float = 0.0):
    """LODParameters::fromCamera / fromCameraWithNearPlane -> (rayOrigSize, rayDirSize)."""
    out = np.zeros(2, np.float32)
    lib().vxo_lod_from_camera(float(fov_y), int(screen_height), float(near_plane), _ptr(out))
    return float(out[0]), float(out[1])


def lod_with_bias(lod, bias: float):
    """LODParameters::withBias."""
    a = np.array(lod, np.float32)
    out = np.zeros(2, np.float32)
    lib().vxo_lod_with_bias(_ptr(a), float(bias), _ptr(out))
    return float(out[0]), float(out[1])


def dxt1_decode_head(head: int) -> np.ndarray:
    out = np.zeros(12, np.float32)
    lib().vxo_dxt1_decode_head(head, _ptr(out))
    return out.reshape(4, 3)


def dxt1_decode_block(block: int) -> np.ndarray:
    out = np.zeros(48, np.float32)
    lib().vxo_dxt1_decode_block(block, _ptr(out))
    return out.reshape(16, 3)


def dxt1_encode_block(colors, indices=None) -> int:
    c = np.ascontiguousarray(colors, dtype=np.float32).reshape(-1, 3)
    idx = None if indices is None else np.ascontiguousarray(indices, dtype=np.int32)
    return int(lib().vxo_dxt1_encode_block(_ptr(c), c.shape[0], _ptr(idx)))


def dxtn_encode_block(normals, indices=None):
    """DXTNormalCompressor::encodeBlockTyped -> (blockA, blockB)."""
    n = np.ascontiguousarray(normals, dtype=np.float32).reshape(-1, 3)
    idx = None if indices is None else np.ascontiguousarray(indices, dtype=np.int32)
    out = np.zeros(2, np.uint64)
    lib().vxo_dxtn_encode_block(_ptr(n), n.shape[0], _ptr(idx), _ptr(out))
    return int(out[0]), int(out[1])


def dxtn_decode_block(block_a: int, block_b: int) -> np.ndarray:
    """DXTNormalCompressor::decodeBlockTyped: 16 unnormalised normals."""
    b = np.array([block_a, block_b], np.uint64)
    out = np.zeros(48, np.float32)
    lib().vxo_dxtn_decode_block(_ptr(b), _ptr(out))
    return out.reshape(16, 3)


def encode_raw_normal(n) -> int:
    a = np.ascontiguousarray(n, dtype=np.float32)
    return int(lib().vxo_encode_raw_normal(_ptr(a)))


def geometric_normals(occ16: np.ndarray) -> np.ndarray:
    """computeGeometricNormal for the 512 voxels of one brick (16 u32 occupancy words)."""
    occ = np.ascontiguousarray(occ16, dtype=np.uint32)
    out = np.zeros(1536, np.float32)
    lib().vxo_geometric_normals(_ptr(occ), _ptr(out))
    return out.reshape(512, 3)


def brick_normals(occ: np.ndarray, threads=0) -> np.ndarray:
    """DXT normal payload of every brick: (bricks, 32, 2) u64 {blockA, blockB}."""
    occ = np.ascontiguousarray(occ, dtype=np.uint32).reshape(-1, 16)
    out = np.zeros((occ.shape[0], 32, 2), np.uint64)
    lib().vxo_brick_normals(_ptr(occ), occ.shape[0], _ptr(out), int(threads))
    return out


def brick_dxt1(rgb: np.ndarray, occ: np.ndarray) -> np.ndarray:
    """DXT1 colour payload (bricks*32 u64) from per-voxel RGB floats and occupancy."""
    rgb = np.ascontiguousarray(rgb, dtype=np.float32)
    occ = np.ascontiguousarray(occ, dtype=np.uint32).reshape(-1, 16)
    out = np.zeros(occ.shape[0] * 32, np.uint64)
    lib().vxo_brick_dxt1(_ptr(rgb), _ptr(occ), occ.shape[0], _ptr(out))
    return out


def hit_normal_dxt(brick_nrm: np.ndarray, brick: int, voxel: int) -> np.ndarray:
    nrm = np.ascontiguousarray(brick_nrm, dtype=np.uint64)
    out = np.zeros(3, np.float32)
    lib().vxo_hit_normal_dxt(_ptr(nrm), brick, voxel, _ptr(out))
    return out


def shade_dxt_normal(color, hit, n_dxt, axis, neg, uv_y) -> int:
    c = np.ascontiguousarray(color, dtype=np.float32)
    n = np.ascontiguousarray(n_dxt, dtype=np.float32)
    return int(lib().vxo_shade_dxt_normal(_ptr(c), int(hit), _ptr(n), int(axis), int(neg), float(uv_y)))


def hit_texel_dxt(brick_dxt: np.ndarray, brick: int, voxel: int) -> np.ndarray:
    out = np.zeros(3, np.float32)
    d = np.ascontiguousarray(brick_dxt, dtype=np.uint64)
    lib().vxo_hit_texel_dxt(_ptr(d), brick, voxel, _ptr(out))
    return out


def camera_rays(pc, width: int, height: int, with_uv_y: bool = False):
    """Primary rays of the shader's camera (getRayDir, RayGeneration.glsl:61-71; uv,
    VoxelRayMarch.comp:453-455).  pc: the 64-byte push-constant block (any object exposing
    the buffer protocol, e.g. a ctypes structure) or 16 floats.  Returns (width*height, 6)
    float32 rows {origin, direction}, row-major from the top row (and uv.y per pixel)."""
    if isinstance(pc, np.ndarray):
        words = np.ascontiguousarray(pc, dtype=np.float32)
    else:
        words = np.frombuffer(bytes(memoryview(pc)), dtype=np.float32).copy()
    assert words.size == 16
    out = np.zeros((width * height, 6), np.float32)
    uv = np.zeros(width * height, np.float32) if with_uv_y else None
    lib().vxo_camera_rays(_ptr(words), width, height, _ptr(out), _ptr(uv))
    return (out, uv) if with_uv_y else out


def material_color(material_id: int, shader: bool = False) -> np.ndarray:
    """MaterialIdToColor (shader=False) or getMaterialColor (shader=True) of one id, 3 float32."""
    out = np.zeros(3, np.float32)
    (lib().vxo_material_color_shader if shader else lib().vxo_material_color_cpu)(int(material_id), _ptr(out))
    return out


def hit_texels_dxt(brick_dxt: np.ndarray, hits: np.ndarray) -> np.ndarray:
    """DXT1 texel (n x 3 float) of every oracle hit record; zeros where brick is 0xFFFFFFFF."""
    d = np.ascontiguousarray(brick_dxt, dtype=np.uint64)
    b = np.ascontiguousarray(hits["brick"], dtype=np.uint32)
    v = np.ascontiguousarray(hits["voxel"], dtype=np.uint32)
    out = np.zeros((b.size, 3), np.float32)
    lib().vxo_hit_texels_dxt(_ptr(d), b.size, _ptr(b), _ptr(v), _ptr(out))
    return out


def shade(color, hit: bool, axis: int, neg: bool, uv_y: float) -> int:
    c = np.ascontiguousarray(color, dtype=np.float32)
    return int(lib().vxo_shade(_ptr(c), int(hit), int(axis), int(neg), float(uv_y)))
