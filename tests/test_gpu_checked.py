"""The bounds-checked build (libvx_checked.so, every device index tested before
its load) on one of every device path (needs a B200): no index goes out of
bounds, and every output equals the default build's bit for bit.  The compacted
batched frame and the compacted shadow pass also equal their all-slots forms."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _run(tmp_path, library):
    out = str(tmp_path / f"{library}.npz")
    env = dict(os.environ, VX_LIBRARY=library)
    r = subprocess.run([sys.executable, os.path.join(HERE, "checked_run.py"), out], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return np.load(out)


def test_checked_build_has_no_violations_and_same_results(tmp_path):
    lib = os.path.join(os.path.dirname(HERE), "vbvs--vixen_b200", "libvx_checked.so")
    if not os.path.exists(lib):
        pytest.fail("libvx_checked.so is not built (make -C vbvs--vixen_b200 checked)")
    checked = _run(tmp_path, "checked")
    default = _run(tmp_path, "default")
    assert int(checked["enabled"][0]) == 1 and int(default["enabled"][0]) == 0
    assert int(checked["violations"][0]) == 0
    for k in default.files:
        if k in ("enabled", "violations"):
            continue
        np.testing.assert_array_equal(checked[k].view(np.uint8), default[k].view(np.uint8), err_msg=k)
    assert int(default["diff_grad_nonzero"][0]) > 0
    # the compacted frame reproduces the eager batched casts
    np.testing.assert_array_equal(default["frame_hits"], default["batch_16"])
    np.testing.assert_array_equal(default["frame_bounce_hits"], default["bounce_hits"])
    np.testing.assert_array_equal(default["shadow_hits"], default["shadow_hits_all_slots"])
