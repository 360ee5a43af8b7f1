"""OBJ vertex assembly on the GPU (nr_scene_load_obj_device) gives the host
reader's meshes bit for bit: vertex order of first use of each (v, vt, vn)
triple, positions, normals (read or generated from face normals in
triangle order), uvs, tangents and triangle indices."""
import numpy as np
import pytest

from nectarrender_b200 import capi, scenes

pytestmark = pytest.mark.gpu


def _both(path):
    spec = scenes.SceneSpec(objects=[], camera={}, meshes=[str(path)])
    host = capi.Scene(spec, build=False).mesh(0)
    dev = capi.Scene(spec, build=False, obj_on_device=True).mesh(0)
    return host, dev


def _same(host, dev):
    for name, a, b in zip(("P", "N", "T", "UV", "tris"), host, dev):
        assert a.shape == b.shape, name
        np.testing.assert_array_equal(a, b, err_msg=name)


def test_mesh_stress_obj_with_normals():
    spec = scenes.mesh_stress(levels=6, res_h=8, res_w=8, spp=1, n_spheres=0, hdri_size=(8, 4))
    host, dev = _both(spec.meshes[0])
    assert host[4].size == 3 * 20 * 4 ** 6
    _same(host, dev)


def test_generated_normals_uvs_quads_and_shared_positions(tmp_path):
    """No vn lines (normals are generated), quads split along the shorter
    diagonal, a polygon fan, negative indices, positions shared by corners
    with different uvs (separate vertices) and a degenerate triangle (its
    face normal is NaN in both)."""
    lines = ["v 0 0 0", "v 1 0 0", "v 1 1 0", "v 0 1 0", "v 0.5 0.5 1", "v 2 0 0", "v 3 0 0"]
    lines += ["vt 0 0", "vt 1 0", "vt 1 1", "vt 0 1", "vt 0.5 0.5"]
    lines += ["f 1/1 2/2 3/3 4/4", "f 1/5 2/2 5/5", "f 2/2 3/3 5/1", "f -4/-1 -3/-2 -5/-3",
              "f 1/1 4/4 5/5 3/3 2/2", "f 2/1 6/2 7/3"]
    p = tmp_path / "mixed.obj"
    p.write_text("\n".join(lines) + "\n")
    _same(*_both(p))


def test_large_random_obj_without_normals(tmp_path):
    rng = np.random.default_rng(3)
    nv, nt, nf = 5000, 700, 60000
    v = rng.uniform(-1, 1, (nv, 3))
    t = rng.uniform(0, 1, (nt, 2))
    f = rng.integers(1, nv + 1, (nf, 3))
    ft = rng.integers(1, nt + 1, (nf, 3))
    out = [f"v {a:.6f} {b:.6f} {c:.6f}" for a, b, c in v]
    out += [f"vt {a:.6f} {b:.6f}" for a, b in t]
    out += [f"f {a}/{x} {b}/{y} {c}/{z}" for (a, b, c), (x, y, z) in zip(f, ft)]
    p = tmp_path / "random.obj"
    p.write_text("\n".join(out) + "\n")
    host, dev = _both(p)
    assert host[0].shape[0] > nv  # positions repeat with different uvs
    _same(host, dev)
