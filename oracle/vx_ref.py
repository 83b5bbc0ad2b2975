"""ctypes binding of the reference build (oracle/_ref/libvx_ref.so).

TEST INFRASTRUCTURE ONLY.  `make -C oracle ref` compiles the reference's own
LaineKarrasOctree::rebuild, castRay / castRayWithLOD, brick DDA and their
dependencies from the reference project's sources, with stand-ins for the two
libraries it needs that are not installed here (glm and gaia-ecs,
oracle/ref_shim/).  The tests use it to pin the oracle to the reference's code:
same voxels, same rays, same results.  available() is False where the library
was not built (no reference sources on that machine).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libvx_ref.so")

# RayHit (SVO/include/ISVOStructure.h:101-112) with the entity as its position
REF_HIT = np.dtype([("t", "<f4"), ("t_exit", "<f4"), ("hit_point", "<f4", 3), ("normal", "<f4", 3),
                    ("hit", "<i4"), ("scale", "<i4"), ("entity_pos", "<f4", 3)])

_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.vxr_build.restype = vp
        L.vxr_build.argtypes = [vp, C.c_uint64, vp, vp, C.c_int, vp, C.c_char_p, C.c_int]
        L.vxr_brick_count.restype = C.c_uint32
        L.vxr_brick_count.argtypes = [vp]
        L.vxr_payloads.argtypes = [vp, vp, vp, vp]
        L.vxr_free.argtypes = [vp]
        L.vxr_node_count.restype = C.c_uint32
        L.vxr_node_count.argtypes = [vp]
        L.vxr_descriptors.argtypes = [vp, vp]
        L.vxr_cast_rays.argtypes = [vp, vp, C.c_uint64, C.c_float, C.c_float, vp, vp]
        _lib = L
    return _lib


class RefOctree:
    """LaineKarrasOctree rebuilt from voxels at world positions (Density 1)."""

    def __init__(self, positions, world_min, world_max, max_levels, materials=None):
        self._keep = [np.ascontiguousarray(np.asarray(positions, np.float32).reshape(-1, 3)),
                      np.ascontiguousarray(world_min, np.float32), np.ascontiguousarray(world_max, np.float32),
                      None if materials is None else np.ascontiguousarray(materials, np.uint32)]
        p, a, b, m = self._keep
        err = C.create_string_buffer(512)
        self._h = lib().vxr_build(p.ctypes.data, p.shape[0], a.ctypes.data, b.ctypes.data, int(max_levels),
                                  None if m is None else m.ctypes.data, err, 512)
        if not self._h:
            raise ValueError(err.value.decode())

    @classmethod
    def from_dense(cls, bits, R, max_levels, material_of=None):
        """Every set voxel of an R^3 bit grid (x fastest, 64 per word) at its integer position;
        material_of(x, y, z) -> material ids (arrays) gives each a Material component."""
        b = np.unpackbits(np.ascontiguousarray(bits, np.uint64).view(np.uint8), bitorder="little")
        idx = np.flatnonzero(b).astype(np.int64)
        x, y, z = idx % R, (idx // R) % R, idx // (R * R)
        pos = np.stack([x, y, z], 1).astype(np.float32)
        mats = None if material_of is None else material_of(x, y, z)
        return cls(pos, (0.0, 0.0, 0.0), (float(R), float(R), float(R)), max_levels, mats)

    def payloads(self):
        """The rebuild's brick payloads: (DXT1 colours bricks*32 u64, DXT normals (bricks, 32, 2)
        u64, material words bricks*512 u32)."""
        B = lib().vxr_brick_count(self._h)
        col = np.zeros(B * 32, np.uint64)
        nrm = np.zeros((B, 32, 2), np.uint64)
        mat = np.zeros(B * 512, np.uint32)
        lib().vxr_payloads(self._h, col.ctypes.data, nrm.ctypes.data, mat.ctypes.data)
        return col, nrm, mat

    def descriptors(self) -> np.ndarray:
        n = lib().vxr_node_count(self._h)
        out = np.zeros(n, np.uint64)
        lib().vxr_descriptors(self._h, out.ctypes.data)
        return out

    def cast_rays(self, rays, t_min=0.0, t_max=3.4028234663852886e38, lod=None):
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        out = np.zeros(r.shape[0], REF_HIT)
        lp = None if lod is None else np.ascontiguousarray(lod, np.float32)
        lib().vxr_cast_rays(self._h, r.ctypes.data, r.shape[0], float(t_min), float(t_max),
                            None if lp is None else lp.ctypes.data, out.ctypes.data)
        return out

    def __del__(self):
        if getattr(self, "_h", None):
            lib().vxr_free(self._h)
            self._h = None
