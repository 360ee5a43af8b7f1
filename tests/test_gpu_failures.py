"""Failure detection on the GPU without a fault: the traversal bounds of a
render (render settings max_traversal_steps and traversal_stack_limit) are
set so small that queries run out of them. The kernels end those queries,
set an error bit (8: step bound, 1: stack overflow) and return; the call
reports NR_ERR_DEVICE with the error word, and the next render on the same
scene is clean and equal to a render that never failed. Also a scene with a
zero-area quad, which renders as the reference does (the quad is never
hit)."""
import re

import numpy as np
import pytest

import oracle
from nectarrender_b200 import capi, last_error, scenes
from tests.gpu_util import frac_close
from tests.test_scene_inputs import zero_area_quad_scene

pytestmark = pytest.mark.gpu
NR_ERR_DEVICE = -7


def _mesh_scene():
    spec = scenes.mesh_stress(levels=4, res_h=64, res_w=64, spp=4, depth=6, n_spheres=16,
                              hdri_size=(128, 64), scene_seed=5)
    return spec, capi.Scene(spec)


def _error_word():
    m = re.search(r"error word 0x([0-9a-f]+)", last_error())
    assert m, last_error()
    return int(m.group(1), 16)


@pytest.mark.parametrize("schedule", [capi.SCHEDULE_WAVEFRONT, capi.SCHEDULE_MEGAKERNEL])
@pytest.mark.parametrize("knob,bit", [("max_traversal_steps", 8), ("traversal_stack_limit", 1)])
def test_traversal_bounds_report_an_error_and_leave_the_device_usable(schedule, knob, bit):
    spec, sc = _mesh_scene()
    bad = capi.Render(sc, schedule=schedule, **{knob: 2})
    for _ in range(2):  # the error word is cleared after each report
        rc = bad.lib.nr_render_samples(bad.h, 1, 2)
        assert rc == NR_ERR_DEVICE
        assert _error_word() & bit
    good = capi.Render(sc, schedule=schedule)
    good.samples(1, 2)
    again = capi.Render(sc, schedule=schedule)
    again.samples(1, 2)
    img = good.layer(0)
    assert np.isfinite(img).all() and img.mean() > 0
    np.testing.assert_array_equal(img, again.layer(0))


def test_zero_area_quad_vs_oracle():
    spec = zero_area_quad_scene(res=48, spp=3)
    r = capi.Render(capi.Scene(spec))
    b, d, n, p = r.sample_layers(1)
    ob, od, on, op, _ = oracle.Oracle().render(spec, 1, mode=0, draw_rtl=capi.device_draw_order())
    assert np.isfinite(b).all()
    assert frac_close(b, ob) >= 0.99
    assert (p == op).mean() >= 0.999
