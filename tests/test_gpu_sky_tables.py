"""HDRI importance-sampling tables built on the GPU (perf mode): the texel
probabilities follow the weight (largest luminance of the 3x3 neighbourhood
times sin(theta)), and the row table composed with each row's column table
puts exactly that probability on every texel."""
import ctypes as C

import numpy as np
import pytest

import oracle
from nectarrender_b200 import capi, scenes

pytestmark = pytest.mark.gpu


def _tables(sc):
    lib = sc.lib
    W, H = C.c_int32(), C.c_int32()
    capi._check(lib.nr_scene_get_sky_tables(sc.h, None, None, None, None, None, C.byref(W),
                                            C.byref(H)), "tables")
    W, H = W.value, H.value
    pdf = np.zeros((H, W), np.float32)
    rp, ra = np.zeros(H, np.float32), np.zeros(H, np.uint32)
    cp, ca = np.zeros((H, W), np.float32), np.zeros((H, W), np.uint32)
    f = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    u = lambda a: a.ctypes.data_as(C.POINTER(C.c_uint32))
    capi._check(lib.nr_scene_get_sky_tables(sc.h, f(pdf), f(rp), u(ra), f(cp), u(ca), None, None),
                "tables")
    return pdf, rp, ra, cp, ca


def _alias_mass(prob, alias):
    n = prob.size
    m = prob.astype(np.float64).copy()
    np.add.at(m, alias, 1.0 - prob.astype(np.float64))
    return m / n


@pytest.mark.parametrize("size", [(256, 128), (512, 256)])
def test_tables_reproduce_the_texel_distribution(size):
    spec = scenes.mesh_stress(levels=3, res_h=8, res_w=8, spp=1, n_spheres=0, hdri_size=size,
                              scene_seed=7)
    sc = capi.Scene(spec)
    pdf, rp, ra, cp, ca = _tables(sc)
    H, W = pdf.shape
    assert (W, H) == size
    # weights from the image: 3x3 maximum of the luminance times sin(theta)
    img = oracle.Oracle().load_hdr(spec.sky["path"]).astype(np.float64)
    lum = np.maximum(0.0, 0.2126 * img[0] + 0.7152 * img[1] + 0.0722 * img[2])
    m = np.zeros_like(lum)
    for dy in (-1, 0, 1):
        rows = np.clip(np.arange(H) + dy, 0, H - 1)
        for dx in (-1, 0, 1):
            m = np.maximum(m, np.roll(lum[rows], -dx, axis=1))
    w = m * np.sin(np.pi * (np.arange(H)[:, None] + 0.5) / H)
    np.testing.assert_allclose(pdf, w / w.sum(), rtol=2e-5, atol=1e-12)
    assert abs(float(pdf.astype(np.float64).sum()) - 1.0) < 1e-5
    # row marginal x column conditional = texel probability
    row_mass = _alias_mass(rp, ra)
    col_mass = np.stack([_alias_mass(cp[y], ca[y]) for y in range(H)])
    implied = row_mass[:, None] * col_mass
    np.testing.assert_allclose(implied, pdf, rtol=1e-4, atol=1e-9)
