"""NR_MODE_PERF (next-event estimation toward lights[0] and the HDRI with
power-heuristic MIS): it converges to the image of the reference's estimator
and reaches a given error with fewer samples."""
import numpy as np
import pytest

from nectarrender_b200 import capi, scenes

pytestmark = pytest.mark.gpu

HI = 4096   # samples of the converged images
LO = 16     # samples of the equal-sample comparison


def _render(sc, mode, first, count, seed=None):
    over = {"mode": mode, "fp64_accumulate": 1}
    if seed is not None:
        over["seed"] = seed
    r = capi.Render(sc, **over)
    r.samples(first, count)
    return r.beauty_fp64()


def _rmse(a, b):
    return float(np.sqrt(np.mean((a - b) ** 2)))


@pytest.mark.parametrize("which", ["cornell_quad_light", "mesh_hdri"])
def test_perf_mode_converges_to_the_reference_estimate(which):
    if which == "cornell_quad_light":
        spec = scenes.cornell(res=32, spp=HI, depth=8, seed=0)
    else:
        spec = scenes.mesh_stress(levels=4, res_h=32, res_w=32, spp=HI, depth=8, n_spheres=16,
                                  hdri_size=(256, 128), scene_seed=5)
    sc = capi.Scene(spec)
    ref = _render(sc, capi.MODE_REFERENCE, 1, HI)
    perf = _render(sc, capi.MODE_PERF, 1, HI)
    assert np.isfinite(perf).all() and (perf >= 0).all()
    # same integral: whole-image means agree within 1%
    for c in range(3):
        assert abs(perf[c].mean() - ref[c].mean()) <= 0.01 * ref[c].mean()
    # and per pixel the difference is at the level of the remaining noise
    # (two independent reference estimates at the same sample count)
    ref2 = _render(sc, capi.MODE_REFERENCE, 1, HI, seed=777)
    assert _rmse(perf, ref) <= 1.5 * _rmse(ref2, ref)

    # equal samples: next-event estimation lowers the error
    lo_ref = _render(sc, capi.MODE_REFERENCE, 1, LO, seed=99)
    lo_perf = _render(sc, capi.MODE_PERF, 1, LO, seed=99)
    assert _rmse(lo_perf, ref) < _rmse(lo_ref, ref)
