"""The small configuration at its own size: the Cornell box at 512x512,
depth 8, seed 0, 64 samples (samples_per_pixel 65), per sample against the
reference's CUDA build (512 is a whole number of its 16x16 blocks), and its
64-sample running mean. Per-sample bar: radiance within 1e-4 relative (floor
1e-3) for at least 99.5% of values, normals for 99.9%; a path that takes
another branch after a last-bit difference differs wholesale, so the bar is a
fraction. The running mean of 64 samples inherits any such path, so it is
held to the reference's own mean in the display domain instead."""
import numpy as np
import pytest

import oracle
from nectarrender_b200 import capi, scenes
from tests.gpu_util import frac_close

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    if not oracle.REF_CUDA_SO.exists():
        pytest.skip("reference CUDA build not present")
    spec = scenes.cornell(res=512, spp=64, depth=8, seed=0)
    sc = capi.Scene(spec)
    return spec, capi.Render(sc), oracle.RefCUDA()


@pytest.mark.parametrize("s", [1, 17, 64])
def test_samples_vs_reference_cuda(setup, s):
    spec, r, rc = setup
    b, d, n, p = r.sample_layers(s)
    rb, rd, rn, _ = rc.render(spec, s, mode=0)
    assert np.isfinite(b).all()
    assert frac_close(b, rb) >= 0.995
    assert frac_close(d, rd) >= 0.995
    assert frac_close(n, rn) >= 0.999


def test_running_mean_of_64_samples(setup):
    spec, r, rc = setup
    r.reset()
    r.render_all()                      # sample indices 1..64, as render() does
    mine = r.layer(0)
    ref, *_ = rc.render(spec, 1, count=64, mode=1)
    disp = lambda x: np.sqrt(np.clip(np.nan_to_num(x), 0.0, 1.0))
    err = float(np.sqrt(np.mean((disp(mine) - disp(ref)) ** 2)))
    assert err <= 2e-3, err
    assert abs(float(mine.mean()) / float(ref.mean()) - 1.0) <= 2e-3
    assert frac_close(mine, ref, rtol=1e-2) >= 0.98
