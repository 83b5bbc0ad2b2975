"""Device noise generator against the host one (needs a B200): identical bits."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("R,spacing,octaves,fill,shell", [(64, 16, 3, 0.1, True), (128, 32, 4, 0.1, True),
                                                         (256, 64, 5, 0.5, False), (128, 16, 2, 0.0, True),
                                                         (64, 8, 1, 1.0, False)])
def test_device_noise_equals_host(vx, cuda, R, spacing, octaves, fill, shell):
    host = vx.synth_noise(R, spacing, octaves, fill, 1234, shell)
    dev = vx.synth_noise_dev(R, spacing, octaves, fill, 1234, shell).cpu().numpy().view(np.uint64)
    np.testing.assert_array_equal(dev, host)
