"""Edge cases of the CUDA integrator (called through the C ABI), per sample:
images of one pixel, one row and one column, a scene without a mesh, a
camera whose every ray misses, paths of depth 1, and a scene at the
1024-object registry limit. Bars as in the parity tests: radiance within 1e-4
relative for at least 99% of values (a path that takes another branch after
a last-ulp difference differs wholesale) and primary-hit ids equal for at
least 99.9% of pixels. Scenes lit by the HDRI are held to the reference's own
CUDA build per sample (both use device fast-math; the host oracle's libm
splits more paths over many bounces) and to the oracle for the primary
hits; the reference CUDA build is run at row counts that are multiples of
16."""
import numpy as np
import pytest

import oracle
from nectarrender_b200 import capi, scenes
from tests.gpu_util import frac_close

pytestmark = pytest.mark.gpu
RTL = 0  # multi-draw arguments evaluated left to right, as the device build does


@pytest.fixture(scope="module")
def orc():
    return oracle.Oracle()


@pytest.fixture(scope="module")
def refcuda():
    if not oracle.REF_CUDA_SO.exists():
        pytest.skip("reference CUDA build not present")
    return oracle.RefCUDA()


def _both(orc, spec, s=1):
    sc = capi.Scene(spec)
    r = capi.Render(sc)
    ours = r.sample_layers(s)
    ref = orc.render(spec, s, mode=0, draw_rtl=RTL)[:4]
    return ours, ref


def _check(ours, ref, frac=0.99):
    (b, d, n, p), (ob, od, on, op) = ours, ref
    assert b.shape == ob.shape
    assert np.isfinite(b).all()
    assert frac_close(b, ob) >= frac
    assert frac_close(d, od) >= frac
    assert frac_close(n, on) >= frac
    assert (p == op).mean() >= 0.999


@pytest.mark.parametrize("h,w", [(1, 1), (1, 53), (41, 1), (3, 5)])
def test_one_pixel_one_row_one_column(orc, h, w):
    spec = scenes.cornell(res=8, spp=2)
    spec.camera["resolution"] = (float(h), float(w))
    ours, ref = _both(orc, spec)
    assert ours[0].shape == (3, h, w)
    _check(ours, ref)


def _check_hdri(orc, refcuda, spec, s=1):
    (b, d, n, p), (ob, od, on, op) = _both(orc, spec, s)
    rb, rd, rn, _ = refcuda.render(spec, s, mode=0)
    assert np.isfinite(b).all()
    assert frac_close(b, rb) >= 0.99
    assert frac_close(n, rn) >= 0.999
    assert (p == op).mean() >= 0.999
    # against the host oracle: within 1e-3 at least as often as the
    # reference's CUDA build is
    assert frac_close(b, ob, rtol=1e-3) >= frac_close(rb, ob, rtol=1e-3) - 0.01


def test_scene_without_a_mesh(orc, refcuda):
    spec = scenes.mesh_stress(levels=2, res_h=32, res_w=48, spp=2, depth=8, n_spheres=40,
                              hdri_size=(128, 64), scene_seed=3)
    spec.objects = [o for o in spec.objects if o["type"] != scenes.MESH]
    spec.meshes = []
    _check_hdri(orc, refcuda, spec)


def test_every_camera_ray_misses(orc):
    spec = scenes.mesh_stress(levels=2, res_h=24, res_w=40, spp=2, depth=4, n_spheres=4,
                              hdri_size=(128, 64), scene_seed=4)
    pitch, yaw, roll = spec.camera["rotation"]
    spec.camera["rotation"] = (pitch, yaw + 180.0, roll)  # facing away from the scene
    spec.camera["position"] = (0.0, 0.2, 9.0)
    ours, ref = _both(orc, spec)
    assert (ours[3] == ref[3]).all()
    assert frac_close(ours[0], ref[0]) >= 0.999  # sky lookups only


@pytest.mark.parametrize("maker", ["cornell", "mesh"])
def test_depth_one(orc, maker):
    if maker == "cornell":
        spec = scenes.cornell(res=32, spp=2, depth=1)
    else:
        spec = scenes.mesh_stress(levels=3, res_h=32, res_w=32, spp=2, depth=1, n_spheres=16,
                                  hdri_size=(128, 64), scene_seed=5)
    _check(*_both(orc, spec))


def test_object_registry_limit(orc, refcuda):
    # one mesh and 1023 spheres: 1024 objects, the registry's limit
    spec = scenes.mesh_stress(levels=2, res_h=32, res_w=32, spp=2, depth=4, n_spheres=1023,
                              hdri_size=(128, 64), scene_seed=6)
    assert len(spec.objects) == 1024
    _check_hdri(orc, refcuda, spec)
