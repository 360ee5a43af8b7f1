"""The launch-shape tuner on a small scene: it times every candidate and
returns the fastest, and the tuned render gives the default render's image.
Knobs that only change launches (traversal kernel, wave length, shading
register budget, material sorting) leave every sample bit-identical; knobs
that reshape the wide BVH (children per node) can only move exact ties, so
the image is held to bit-equality on all but a sliver of values there."""
import json

import numpy as np
import pytest

from nectarrender_b200 import autotune, capi, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def spec():
    return scenes.mesh_stress(levels=5, res_h=96, res_w=96, spp=8, depth=8, n_spheres=24,
                              hdri_size=(256, 128), scene_seed=6)


def _image(spec, t: autotune.Tuning):
    sc = capi.Scene(spec, **t.scene_overrides())
    r = capi.Render(sc, **t.render_overrides())
    r.samples(1, 4)
    return r.layer(0)


def test_tune_picks_the_fastest_candidate(spec, tmp_path):
    t = autotune.tune(spec, samples=2, reps=1, leaves=((1, 1),), variants=(574, 14),
                      waves=(0, 2), shades=(5, 6), sorts=(1,), megakernel=False,
                      widths=((8, 8), (4, 4)))
    assert len(t.table) == 2 * 2 * 2 * 2
    assert t.ms_per_sample == min(row["ms_per_sample"] for row in t.table) > 0
    path = tmp_path / "tuning.json"
    autotune.save(path, spec, t)
    assert autotune.load(path, spec).render_overrides() == t.render_overrides()
    json.loads(path.read_text())
    base = _image(spec, autotune.Tuning())
    tuned = _image(spec, t)
    if (t.mesh_width, t.tlas_width) == (8, 8):
        np.testing.assert_array_equal(tuned, base)
    else:
        assert (tuned == base).mean() >= 0.999


@pytest.mark.parametrize("variant,wave,shade", [(14, 2, 5), (515, 0, 6), (5, 4, 5), (564, 0, 6),
                                                (84, 2, 6)])
def test_launch_knobs_leave_samples_bit_identical(spec, variant, wave, shade):
    base = _image(spec, autotune.Tuning())
    t = autotune.Tuning(extend_variant=variant, samples_per_wave=wave, shade_variant=shade)
    np.testing.assert_array_equal(_image(spec, t), base)


def test_narrow_trees_render_the_same_hits(spec):
    base = _image(spec, autotune.Tuning())
    t = autotune.Tuning(mesh_width=4, tlas_width=4)
    img = _image(spec, t)
    assert (img == base).mean() >= 0.999
    st4 = capi.Scene(spec, mesh_width=4, tlas_width=4).stats()
    st8 = capi.Scene(spec).stats()
    assert st4["wide_nodes"] > st8["wide_nodes"]          # smaller nodes, more of them
    # the same binary tree (its cost summed on the GPU in another order)
    assert st4["sah_cost_binary"] == pytest.approx(st8["sah_cost_binary"], rel=1e-9)
