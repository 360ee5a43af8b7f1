"""The oracle's viewport preview, picking ray and selection outline against
the reference's own camera, traversal, material and grid code compiled for
the host (oracle/_ref/libref_cpu.so), and against the committed fixture."""
from pathlib import Path

import numpy as np
import pytest

import oracle
from nectarrender_b200 import scenes

GOLDEN = Path(__file__).parent / "golden"


@pytest.fixture(scope="module")
def orc():
    oracle.build(reference_root="")
    return oracle.Oracle()


def _specs():
    return {"cornell": scenes.cornell(res=24, spp=3)}  # the fixture's scene


def test_viewport_fixture(orc):
    g = np.load(GOLDEN / "viewport24.npz")
    h = orc.open_scene(_specs()["cornell"], draw_rtl=0)
    for grid in (0, 1):
        b, d, n = h.viewport(bool(grid))
        np.testing.assert_array_equal(b, g[f"beauty_grid{grid}"])
        np.testing.assert_array_equal(d, g[f"diffuse_grid{grid}"])
        np.testing.assert_array_equal(n, g[f"normal_grid{grid}"])
    for k, (u, v) in enumerate(g["pick_uv"]):
        p = h.pick(float(u), float(v))
        assert int(p["hit"]) == int(g["pick_hit"][k])
        if p["hit"]:
            assert p["object_id"] == int(g["pick_obj"][k])
            assert np.float32(p["t"]) == g["pick_t"][k]
    oid = int(g["mask_object"])
    np.testing.assert_array_equal(h.selection_mask(oid, 2), g["mask_r2"])


@pytest.mark.skipif(not oracle.REF_CPU_SO.exists(), reason="reference host build not present")
def test_viewport_matches_reference_live(orc):
    ref = oracle.RefCPU()
    spec = scenes.mesh_stress(levels=3, res_h=40, res_w=40, spp=2, depth=4, n_spheres=8,
                              hdri_size=(64, 32), scene_seed=2)
    ho, hr = orc.open_scene(spec, draw_rtl=0), ref.open_scene(spec, draw_rtl=1)
    for grid in (True, False):
        for a, b in zip(ho.viewport(grid), hr.viewport(grid)):
            np.testing.assert_array_equal(a, b)
    rng = np.random.default_rng(3)
    for u, v in rng.uniform(0.02, 0.98, size=(20, 2)):
        assert ho.pick(u, v) == hr.pick(u, v)
    oid = hr.pick(0.5, 0.5)["object_id"]
    np.testing.assert_array_equal(ho.selection_mask(oid, 3), hr.selection_mask(oid, 3))
