"""Seeded scene generators and file formats."""
import numpy as np

import oracle
from nectarrender_b200 import scenes


def test_icosphere_counts():
    for lv in range(0, 4):
        v, f = scenes.icosphere(lv)
        assert len(f) == 20 * 4 ** lv
        assert len(v) == 10 * 4 ** lv + 2
        assert np.allclose(np.linalg.norm(v, axis=1), 1.0)


def test_displacement_bounds_and_determinism():
    v1, f1, n1 = scenes.displaced_icosphere(3, seed=5)
    v2, f2, n2 = scenes.displaced_icosphere(3, seed=5)
    assert np.array_equal(v1, v2) and np.array_equal(f1, f2)
    r = np.linalg.norm(v1, axis=1)
    assert r.min() >= 0.95 - 1e-9 and r.max() <= 1.05 + 1e-9
    assert np.allclose(np.linalg.norm(n1, axis=1), 1.0)


def test_hdr_roundtrip_through_oracle_reader(tmp_path):
    rgb = scenes.procedural_hdri(64, 32, seed=2)
    p = tmp_path / "s.hdr"
    scenes.write_hdr(p, rgb)
    img = oracle.Oracle().load_hdr(str(p))
    assert img.shape == (3, 32, 64)
    back = np.transpose(img, (1, 2, 0))
    # RGBE keeps 8 mantissa bits of the largest channel
    assert np.all(np.abs(back - rgb) <= rgb.max(axis=2, keepdims=True) / 128 + 1e-30)


def test_cornell_layout():
    spec = scenes.cornell(res=32, spp=4)
    assert spec.camera["samples_per_pixel"] == 5   # renders samples 1..4
    assert spec.objects[-1]["type"] == scenes.LIGHT
    assert sum(o["type"] == scenes.SPHERE for o in spec.objects) == 3


def test_mesh_stress_spheres_do_not_overlap():
    spec = scenes.mesh_stress(levels=1, res_h=8, res_w=8, spp=1, n_spheres=64, hdri_size=(16, 8),
                              scene_seed=9)
    sph = [(np.array(o["position"]), o["radius"]) for o in spec.objects if o["type"] == scenes.SPHERE]
    assert len(sph) == 64
    for i, (p, r) in enumerate(sph):
        assert 0.05 <= r <= 0.3
        assert np.linalg.norm(p) >= 1.06 + r
        for q, s in sph[:i]:
            assert np.linalg.norm(p - q) >= r + s


def test_spec_json_roundtrip_keeps_images_and_texture_slots():
    import json
    import numpy as np
    spec = scenes.cornell_textured_mesh(res=16, spp=2)
    d = json.loads(json.dumps(scenes.spec_to_json(spec)))
    back = scenes.spec_from_json(d)
    assert len(back.images) == len(spec.images)
    for a, b in zip(spec.images, back.images):
        assert b.dtype == np.uint8 and np.array_equal(a, b)
    assert back.meshes == spec.meshes
    for o, p in zip(spec.objects, back.objects):
        assert o["material"]["tex"] == p["material"]["tex"]
    assert scenes.spec_to_json(back) == d


def test_uv_sphere_mesh():
    import numpy as np
    v, f, n, uv = scenes.uv_sphere(8, 16)
    assert np.allclose(np.linalg.norm(v, axis=1), 1.0)
    assert uv.min() >= 0.0 and uv.max() <= 1.0
    assert f.max() < len(v) and len(f) == 2 * 8 * 16 - 2 * 16  # the pole rows lose one triangle per quad
