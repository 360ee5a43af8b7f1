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


def test_band_matches_oracle(full):
    spec, sc, r = full
    b, d, n, p = r.sample_layers(3)
    h = oracle.Oracle().open_scene(spec, draw_rtl=0)
    ob, od, on, op, _ = h.render(3, 1, mode=0, rows=(500, 540))
    band = slice(500, 540)
    assert (p[band] == op[band]).mean() >= 0.999
    # Unit normals, absolute bar. Grazing sphere hits amplify the device's
    # fused multiply-adds in the quadratic's discriminant (the oracle is host
    # code without contraction) into ~1e-4 moves of the hit point; the
    # ulp-level bar is against the reference's CUDA build in the parity tests.
    dn = np.abs(n[:, band] - on[:, band])
    assert (dn <= 2e-4).mean() >= 0.99
    assert float(np.median(dn)) <= 1e-6
    # host libm (oracle) versus device fast-math moves HDRI lookups by ulps;
    # the tight per-sample bar is against the reference's CUDA build
    assert frac_close(b[:, band], ob[:, band], rtol=1e-3) >= 0.97
