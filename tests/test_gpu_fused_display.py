"""Fused display (nr_render_set_fused_display): the accumulate pass writes
the beauty layer's display bytes, and a readback with the same config copies
them; the bytes equal the separate display pass, and any change that the
fused bytes do not reflect (another config, a reset, a raw-sample call)
falls back to the display pass."""
import ctypes as C

import numpy as np
import pytest

from nectarrender_b200 import capi, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene():
    spec = scenes.mesh_stress(levels=4, res_h=48, res_w=64, spp=9, depth=8, n_spheres=16,
                              hdri_size=(128, 64), scene_seed=5)
    return capi.Scene(spec)


@pytest.mark.parametrize("cfg", [dict(), dict(white_balance=True, temperature=5000.0, tint=4.0),
                                 dict(method=2, alpha=0.7), dict(method=1, white_point=2.5)])
def test_fused_bytes_equal_the_display_pass(scene, cfg):
    sc = capi.stream_config(**cfg)
    fused, plain = capi.Render(scene), capi.Render(scene)
    capi._check(fused.lib.nr_render_set_fused_display(fused.h, C.byref(sc)), "fused")
    for first, count in ((1, 3), (4, 5)):
        fused.samples(first, count)
        plain.samples(first, count)
        np.testing.assert_array_equal(fused.readback(0, sc), plain.readback(0, sc))


def test_stale_fused_bytes_are_not_used(scene):
    sc = capi.stream_config()
    other = capi.stream_config(method=2)
    r, plain = capi.Render(scene), capi.Render(scene)
    capi._check(r.lib.nr_render_set_fused_display(r.h, C.byref(sc)), "fused")
    r.samples(1, 4)
    plain.samples(1, 4)
    np.testing.assert_array_equal(r.readback(0, other), plain.readback(0, other))  # other config
    r.reset()
    plain.reset()
    np.testing.assert_array_equal(r.readback(0, sc), plain.readback(0, sc))  # after a reset
    r.samples(1, 2)
    r.sample_layers(3)  # raw samples overwrite the layers
    plain.samples(1, 2)
    plain.sample_layers(3)
    np.testing.assert_array_equal(r.readback(0, sc), plain.readback(0, sc))
    capi._check(r.lib.nr_render_set_fused_display(r.h, None), "off")
    r.samples(4, 2)
    plain.samples(4, 2)
    np.testing.assert_array_equal(r.readback(0, sc), plain.readback(0, sc))
