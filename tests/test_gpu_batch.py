"""Several scenes rendered in one nr_render_samples_batch call equal the
same scenes rendered one after another."""
import numpy as np
import pytest

from nectarrender_b200 import capi, scenes

pytestmark = pytest.mark.gpu


def test_batch_equals_sequential():
    specs = scenes.scene_set(4, seed=3, max_level=4)
    scs = [capi.Scene(s) for s in specs]
    seq = [capi.Render(sc) for sc in scs]
    bat = [capi.Render(sc) for sc in scs]
    counts = [min(4, s.camera["samples_per_pixel"] - 1) for s in specs]
    for r, c in zip(seq, counts):
        r.samples(1, c)
    capi.render_batch(bat, [1] * len(bat), counts)
    for a, b in zip(seq, bat):
        for layer in (0, 1, 4):
            np.testing.assert_array_equal(a.layer(layer), b.layer(layer))
    # a second batch continues the running means
    capi.render_batch(bat, [c + 1 for c in counts], [1] * len(bat))
    for r, c in zip(seq, counts):
        r.samples(c + 1, 1)
    for a, b in zip(seq, bat):
        np.testing.assert_array_equal(a.layer(0), b.layer(0))


def test_batch_rejects_duplicates_and_bad_indices():
    spec = scenes.cornell(res=32, spp=2, depth=2)
    r = capi.Render(capi.Scene(spec))
    with pytest.raises(RuntimeError, match="twice"):
        capi.render_batch([r, r], [1, 1], [1, 1])
    with pytest.raises(RuntimeError, match="beyond"):
        capi.render_batch([r], [1], [5])
