"""Primary-ray generation (row A1): the library's host form vx_camera_rays against the
oracle's independent restatement of getRayDir (shaders/RayGeneration.glsl:61-71) and the
pixel uv of VoxelRayMarch.comp:453-455, bit for bit.  CPU only (the device form and the
render kernel's in-kernel rays are checked in test_gpu_parity.py)."""
import numpy as np
import pytest


@pytest.mark.parametrize("fov,w,h", [(60.0, 512, 512), (70.0, 1920, 1080), (45.0, 7, 5), (120.0, 33, 400)])
def test_host_camera_rays_equal_oracle(vx, vo, fov, w, h):
    from vx_b200 import workloads as W
    rng = np.random.default_rng(w * 1000 + h)
    for _ in range(3):
        pos = rng.uniform(-100, 1100, 3)
        d = rng.normal(size=3)
        pc = W.look_camera(pos, d, fov, w, h)
        want, uv_y = vo.camera_rays(pc, w, h, with_uv_y=True)
        got = vx.camera_rays(pc, w, h)
        np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
    # uv.y of row y is (y + 0.5) / h, the value the miss colour reads
    rows = np.arange(w * h) // w
    np.testing.assert_array_equal(uv_y, ((rows.astype(np.float32) + np.float32(0.5)) / np.float32(h)))


def test_benchmark_cameras_equal_oracle(vx, vo):
    """The cameras of the benchmark frames: cfg1's face-centre camera, a cfg2-style seeded camera
    and cfg3's urban camera, at their full resolutions."""
    from vx_b200 import workloads as W
    bits = np.zeros(64 * 64, np.uint64)
    cams = [(W.look_camera([128.5, 128.5, 1.5], [0, 0, 1], 60.0, 512, 512), 512, 512),
            (W.empty_voxel_camera(bits, 64, 2, 70.0, 1920, 1080), 1920, 1080),
            (W.look_camera([1024.0, 1843.2, -512.0], [0.05, -0.45, 1.0], 60.0, 3840, 2160), 3840, 2160)]
    for pc, w, h in cams:
        np.testing.assert_array_equal(vx.camera_rays(pc, w, h).view(np.uint32),
                                      vo.camera_rays(pc, w, h).view(np.uint32))
