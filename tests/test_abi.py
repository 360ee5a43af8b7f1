"""The C-ABI library loads, exports every declared symbol, and reports
argument and state errors without touching a GPU."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import nectarrender_b200 as nb
from nectarrender_b200 import capi, scenes

HEADER = Path(__file__).resolve().parents[1] / "include" / "nectar_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(nr_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    lib = nb.library()
    names = declared_symbols()
    assert len(names) >= 39
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(capi.EXPORTS) == names


def test_abi_version():
    assert nb.library().nr_abi_version() == 1


def test_draw_order_default_is_device_left_to_right():
    lib = nb.library()
    assert lib.nr_device_draw_order() == 0
    lib.nr_set_draw_order(1)
    assert lib.nr_device_draw_order() == 1
    lib.nr_set_draw_order(0)


def test_scene_registry_errors():
    lib = nb.library()
    h = C.c_void_p()
    assert lib.nr_scene_create(C.byref(h)) == 0
    d = capi.object_desc(scenes.obj(scenes.QUAD, None), material=99)
    assert lib.nr_scene_add_object(h, C.byref(d), None) == -1  # unknown material
    assert b"material" in nb.library().nr_last_error()
    m = capi.material_desc(scenes.lambertian((0.5, 0.5, 0.5)))
    mid = C.c_uint32()
    assert lib.nr_scene_add_material(h, C.byref(m), C.byref(mid)) == 0 and mid.value == 1
    d = capi.object_desc(scenes.obj(scenes.QUAD, None), material=1)
    for _ in range(1024):
        assert lib.nr_scene_add_object(h, C.byref(d), None) == 0
    assert lib.nr_scene_add_object(h, C.byref(d), None) == -3  # registry limit (1024)
    assert b"1024" in nb.library().nr_last_error()
    lib.nr_scene_destroy(h)


def test_empty_scene_and_missing_files():
    lib = nb.library()
    h = C.c_void_p()
    lib.nr_scene_create(C.byref(h))
    assert lib.nr_scene_build(h) == -1
    assert b"empty" in nb.library().nr_last_error()
    assert lib.nr_scene_load_obj(h, b"/nonexistent.obj", None) == -4
    assert lib.nr_scene_load_hdr(h, b"/nonexistent.hdr", C.c_float(0), C.c_float(1)) == -4
    lib.nr_scene_destroy(h)


@pytest.mark.skipif(nb.device_count() > 0, reason="checks the no-device path")
def test_build_without_device_fails_loudly():
    spec = scenes.cornell(res=8, spp=1)
    with pytest.raises(RuntimeError, match="no CUDA device"):
        capi.Scene(spec)


def test_product_obj_reader_matches_reference_fixture():
    from tests.golden.make_golden import HERE as GOLDEN, local_mesh_spec
    g = np.load(GOLDEN / "mesh_small.npz")
    spec = local_mesh_spec()
    sc = capi.Scene(spec, build=False)
    P, N, T, UV, tris = sc.mesh(0)
    for a, k in zip((P, N, T, UV, tris), ("obj_P", "obj_N", "obj_T", "obj_UV", "obj_tris")):
        assert np.array_equal(a, g[k]), k


def test_product_obj_reader_in_chunks_matches_the_oracle(tmp_path):
    """A multi-megabyte OBJ is parsed by several host threads in line-aligned
    chunks; the mesh equals the oracle's single-pass reader (and the
    reference's own, when its build is present), including relative indices
    and quads that refer to vertices of earlier chunks."""
    import oracle
    v, f, n = scenes.displaced_icosphere(6, seed=4)
    p = tmp_path / "big.obj"
    scenes.write_obj(p, v, f, n)
    with open(p, "a") as fh:  # faces whose indices reach back across the chunks
        fh.write("f -1//-1 -2//-2 -3//-3 -4//-4\nf 1//1 2//2 3//3 4//4\n")
    assert p.stat().st_size > 4 << 20
    spec = scenes.SceneSpec(objects=[], camera={}, meshes=[str(p)])
    got = capi.Scene(spec, build=False).mesh(0)
    refs = [oracle.Oracle().load_obj(str(p))]
    if oracle.REF_CPU_SO.exists():
        refs.append(oracle.RefCPU().load_obj(str(p)))
    for ref in refs:
        for name, a, b in zip(("P", "N", "T", "UV", "tris"), got, ref):
            np.testing.assert_array_equal(a, np.asarray(b).reshape(a.shape), err_msg=name)


@pytest.mark.parametrize("verts,expected", [
    ("v 0 0 0\nv 2 0 0\nv 1 1 0\nv -1 1 0\n", [0, 1, 2, 0, 2, 3]),   # 0-2 shorter
    ("v 0 0 0\nv 2 0 0\nv 2 1 0\nv 1 1 0\n", [0, 1, 2, 1, 3, 2]),    # 1-3 shorter
])
def test_obj_quads_split_like_tinyobjloader(tmp_path, verts, expected):
    import oracle
    p = tmp_path / "quad.obj"
    p.write_text(verts + "f 1 2 3 4\n")
    spec = scenes.SceneSpec(objects=[], camera={}, meshes=[str(p)])
    sc = capi.Scene(spec, build=False)
    *_, tris = sc.mesh(0)
    assert tris.tolist() == expected
    if oracle.REF_CPU_SO.exists():
        *_, ref_tris = oracle.RefCPU().load_obj(str(p))
        assert ref_tris.tolist() == expected


def test_checker_libraries_export_their_header():
    """liboracle.so (and the reference builds, when present) export every
    function oracle/oracle.h declares for them."""
    import oracle
    text = (Path(oracle.__file__).parent / "oracle.h").read_text()
    for path, prefix in ((oracle.ORACLE_SO, "oracle_"), (oracle.REF_CPU_SO, "refcpu_"),
                         (oracle.REF_CUDA_SO, "refcuda_")):
        if not path.exists():
            continue
        lib = C.CDLL(str(path))
        for name in sorted(set(re.findall(rf"\b({prefix}[a-z0-9_]+)\s*\(", text))):
            assert hasattr(lib, name), (path.name, name)
