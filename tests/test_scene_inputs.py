"""Scene inputs the library refuses on the host, before any GPU work: an OBJ
file with a valid header but no faces, non-finite vertex positions (from an
OBJ file or from arrays), and non-finite object transforms. No GPU is
needed: these checks run before a device is touched."""
import ctypes as C

import numpy as np
import pytest

import nectarrender_b200 as nb
from nectarrender_b200 import capi, scenes

NR_ERR_INVALID = -1


@pytest.fixture()
def scene():
    lib = nb.library()
    h = C.c_void_p()
    assert lib.nr_scene_create(C.byref(h)) == 0
    yield lib, h
    lib.nr_scene_destroy(h)


def _write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p).encode()


@pytest.mark.parametrize("loader", ["nr_scene_load_obj", "nr_scene_load_obj_device"])
def test_obj_without_faces_is_refused(scene, tmp_path, loader):
    lib, h = scene
    path = _write(tmp_path, "empty.obj", "# exported\no empty\nv 0 0 0\nv 1 0 0\nv 0 1 0\n")
    assert getattr(lib, loader)(h, path, None) == NR_ERR_INVALID
    assert "no faces" in nb.last_error()


@pytest.mark.parametrize("loader", ["nr_scene_load_obj", "nr_scene_load_obj_device"])
def test_obj_with_a_nan_vertex_is_refused(scene, tmp_path, loader):
    lib, h = scene
    path = _write(tmp_path, "nan.obj", "v 0 0 0\nv 1 nan 0\nv 0 1 0\nf 1 2 3\n")
    assert getattr(lib, loader)(h, path, None) == NR_ERR_INVALID
    assert "non-finite" in nb.last_error()


def test_mesh_arrays_with_inf_are_refused(scene):
    lib, h = scene
    P = np.array([0, 0, 0, 1, 0, 0, 0, np.inf, 0], np.float32)
    T = np.array([0, 1, 2], np.uint32)
    fp = P.ctypes.data_as(C.POINTER(C.c_float))
    rc = lib.nr_scene_add_mesh(h, fp, None, None, None, 3, T.ctypes.data_as(C.POINTER(C.c_uint32)),
                               1, None)
    assert rc == NR_ERR_INVALID and "non-finite" in nb.last_error()
    P[7] = 1.0
    rc = lib.nr_scene_add_mesh(h, fp, None, None, None, 3, T.ctypes.data_as(C.POINTER(C.c_uint32)),
                               1, None)
    assert rc == 0


@pytest.mark.parametrize("field,value", [("position", (0.0, float("nan"), 0.0)),
                                         ("scale", (1.0, float("inf"), 1.0)),
                                         ("radius", float("nan"))])
def test_non_finite_transforms_are_refused(scene, field, value):
    lib, h = scene
    o = scenes.obj(scenes.SPHERE, scenes.lambertian((0.5, 0.5, 0.5)), radius=0.5)
    o[field] = value
    d = capi.object_desc(o, 0)
    assert lib.nr_scene_add_object(h, C.byref(d), None) == NR_ERR_INVALID
    assert "non-finite" in nb.last_error()


def zero_area_quad_scene(res=32, spp=2):
    """The Cornell box with a quad of zero width standing in it."""
    spec = scenes.cornell(res=res, spp=spp)
    spec.objects.insert(5, scenes.obj(scenes.QUAD, scenes.lambertian((0.9, 0.2, 0.2)), (0, 0, 0),
                                      (0, 30, 0), (0.0, 1.0, 0.6)))
    return spec


def test_zero_area_quad_oracle_matches_reference():
    import oracle
    if not oracle.REF_CPU_SO.exists():
        pytest.skip("reference host build not present")
    spec = zero_area_quad_scene()
    b, d, n, p, _ = oracle.Oracle().render(spec, 1, mode=0, draw_rtl=1)
    rb, rd, rn, rp, _ = oracle.RefCPU().render(spec, 1, mode=0)
    assert np.isfinite(b).all()
    np.testing.assert_array_equal(b, rb)
    np.testing.assert_array_equal(p, rp)
