"""The full mesh-stress configuration: 1,310,720 triangles, 1920x1080,
depth 12, HDRI; size-independent properties and agreement with the oracle on
a band of rows."""
import numpy as np
import pytest

import oracle
from nectarrender_b200 import capi, scenes
from tests.gpu_util import frac_close

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def full():
    spec = scenes.mesh_stress()
    sc = capi.Scene(spec)
    return spec, sc, capi.Render(sc)


def test_render_and_counters(full):
    spec, sc, r = full
    r.counters(True)
    r.samples(1, 2)
    c = r.last_counters()
    r.counters(False)
    assert c["paths"] == 2 * 1920 * 1080
    assert c["rays"] >= c["paths"]
    img = r.layer(0)
    assert np.isfinite(img).all() and img.mean() > 0


@pytest.fixture(scope="module")
def full_1088():
    # The reference's 2D kernels have no bounds guard and read past the
    # layers unless the rows are a multiple of their 16-row tiles, so the
    # comparison with its CUDA build uses 1088 rows.
    spec = scenes.mesh_stress(res_h=1088)
    sc = capi.Scene(spec)
    return spec, sc, capi.Render(sc)


def test_full_frame_matches_reference_cuda(full_1088):
    spec, sc, r = full_1088
    b, d, n, p = r.sample_layers(3)
    rb, rd, rn, _ = oracle.RefCUDA().render(spec, 3, mode=0)
    # per-sample agreement within 1e-4 over 12 bounces of 2.1 M paths
    assert frac_close(b, rb) >= 0.98
    assert frac_close(d, rd) >= 0.999
    assert frac_close(n, rn) >= 0.999


def test_band_matches_oracle(full_1088):
    spec, sc, r = full_1088
    b, d, n, p = r.sample_layers(3)
    h = oracle.Oracle().open_scene(spec, draw_rtl=0)
    ob, od, on, op, _ = h.render(3, 1, mode=0, rows=(500, 540))
    band = slice(500, 540)
    assert (p[band] == op[band]).mean() >= 0.999
    # Unit normals, absolute bar. Grazing sphere hits amplify the device's
    # fused multiply-adds in the quadratic's discriminant (the oracle is host
    # code without contraction) into ~1e-4 moves of the hit point.
    dn = np.abs(n[:, band] - on[:, band])
    assert (dn <= 2e-4).mean() >= 0.99
    assert float(np.median(dn)) <= 1e-6
    # Host libm against device fast-math splits some of the 12-bounce paths;
    # this build agrees with the host oracle as well as the reference's own
    # CUDA build does (both about 0.90 of values within 1e-3 on this band).
    rb, *_ = oracle.RefCUDA().render(spec, 3, mode=0)
    ref_agree = frac_close(rb[:, band], ob[:, band], rtol=1e-3)
    assert frac_close(b[:, band], ob[:, band], rtol=1e-3) >= ref_agree - 0.01
