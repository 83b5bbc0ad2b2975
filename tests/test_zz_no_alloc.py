"""vx_cast_batch_noalloc, the batched cast that allocates no device memory
(needs a B200).

Some callers cannot allocate device memory: an application that owns a fixed
device-memory budget, or a frame loop that cannot take cudaMalloc's implicit
device synchronisation.  This entry point takes the scenes directly and keeps
its scratch (task counter, scene table) in a static device array.  The test
calls it through the C ABI twice in a row, with different rays, and checks
both results against the allocating entry point vx_cast_batch, bit for bit
(the tolerance of every parity test here).  This file is collected last so a
run that stops at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_matches_batched_on_two_calls(vx, cuda):
    import torch
    from vx_b200 import workloads as W
    specs = W.config4_specs(6, seed=21, r_range=(6, 7.4), res_lo=(48, 40), res_hi=(160, 96))
    wls = [W.build_spec(s) for s in specs]
    scenes = [vx.Scene(w.scene) for w in wls]
    rays = [w.rays() for w in wls]
    begin = np.concatenate([[0], np.cumsum([r.shape[0] for r in rays])]).astype(np.int32)
    n = int(begin[-1])
    d_rays = torch.from_numpy(np.concatenate(rays)).cuda()
    d_begin = torch.from_numpy(begin).cuda()
    d_bbegin = torch.from_numpy(2 * begin).cuda()
    batch = vx.Batch(scenes)
    ref1 = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    batch.cast(d_rays, d_begin, ref1)
    bounce = torch.zeros((2 * n, 6), dtype=torch.float32, device="cuda")
    vx.spawn_bounce_rays(d_rays, ref1, 5, bounce)
    ref2 = torch.zeros((2 * n, 4), dtype=torch.int32, device="cuda")
    batch.cast(bounce, d_bbegin, ref2)
    torch.cuda.synchronize()

    got1 = torch.full((n, 4), -1, dtype=torch.int32, device="cuda")
    got2 = torch.full((2 * n, 4), -1, dtype=torch.int32, device="cuda")
    vx.cast_batch_noalloc(scenes, d_rays, d_begin, got1)     # first call: primary rays
    vx.cast_batch_noalloc(scenes, bounce, d_bbegin, got2)    # second call: bounce rays
    torch.cuda.synchronize()
    np.testing.assert_array_equal(got1.cpu().numpy(), ref1.cpu().numpy())
    np.testing.assert_array_equal(got2.cpu().numpy(), ref2.cpu().numpy())
    assert int(np.count_nonzero(got1.cpu().numpy().view(vx.HIT_DTYPE)["flags"] & 1)) > 0


def test_noalloc_rejects_more_scenes_than_its_scratch_holds(vx, cuda):
    import torch
    from vx_b200 import workloads as W
    s = vx.Scene(W.config1(R=64, width=8, height=8).scene)
    k = vx.VX_NOALLOC_MAX_SCENES + 1
    arr = (C.c_void_p * k)(*([s.handle.value] * k))
    begin = torch.zeros(k + 1, dtype=torch.int32, device="cuda")
    rays = torch.zeros((1, 6), dtype=torch.float32, device="cuda")
    hits = torch.zeros((1, 4), dtype=torch.int32, device="cuda")
    rc = vx.lib().vx_cast_batch_noalloc(arr, k, C.c_void_p(rays.data_ptr()), C.c_void_p(begin.data_ptr()), 0,
                                        0.0, 1.0, C.c_void_p(hits.data_ptr()), None)
    assert rc == -3
    assert "scene count" in vx.lib().vx_last_error_string().decode()
