"""nr_render_samples_static renders from a library-owned static device buffer
and allocates nothing during the call. Its layers must equal those of
nr_render_samples on the same scene, over two calls in a row. Named to be
collected last, so it also runs after every other GPU test in the process."""
import numpy as np
import pytest

from nectarrender_b200 import capi, last_error, scenes

pytestmark = pytest.mark.gpu

NR_ERR_LIMIT = -3
NR_ERR_STATE = -6
NR_STATIC_WAVE_PATHS = 270528
LAYERS = (0, 1, 4)  # beauty, diffuse, world normal


TAIL_OFF = 0xFFFFFFFF


def _pair(spec, **cfg):
    # The static entry point never hands a wave's last bounces to the
    # per-path tail kernel (whose stack could make the driver grow its
    # local-memory reservation); the allocating render is set up the same
    # way, so that both run the same kernels.
    sc = capi.Scene(spec)
    return sc, capi.Render(sc, tail_max_paths=TAIL_OFF, **cfg), capi.Render(sc, **cfg)


@pytest.mark.parametrize("which", ["cornell", "mesh_hdri"])
def test_static_matches_allocating_entry_point(which):
    if which == "cornell":
        spec = scenes.cornell(res=128, spp=8, depth=8, seed=0)
    else:
        spec = scenes.mesh_stress(levels=4, res_h=96, res_w=96, spp=8, depth=12, n_spheres=16,
                                  hdri_size=(128, 64), scene_seed=3)
    sc, alloc, static = _pair(spec)
    for first, count in ((1, 3), (4, 4)):
        alloc.samples(first, count)
        rc = static.lib.nr_render_samples_static(static.h, first, count)
        assert rc == 0, last_error()
        for layer in LAYERS:
            np.testing.assert_allclose(static.layer(layer), alloc.layer(layer),
                                       rtol=1e-6, atol=1e-7)


def test_static_waves_split_at_the_buffer_capacity():
    # 384x384 = 147,456 pixels: one sample index per static wave, while the
    # allocating path puts four in one wave; the layers still agree
    spec = scenes.cornell(res=384, spp=4, depth=6, seed=1)
    sc, alloc, static = _pair(spec, samples_per_wave=4)
    alloc.samples(1, 4)
    assert static.lib.nr_render_samples_static(static.h, 1, 4) == 0, last_error()
    for layer in LAYERS:
        np.testing.assert_allclose(static.layer(layer), alloc.layer(layer), rtol=1e-6, atol=1e-7)


def test_static_rejects_images_beyond_the_buffer():
    spec = scenes.cornell(res=544, spp=2, depth=4, seed=0)  # 295,936 pixels
    sc = capi.Scene(spec)
    r = capi.Render(sc)
    assert r.lib.nr_render_samples_static(r.h, 1, 1) == NR_ERR_LIMIT
    msg = last_error()
    assert str(NR_STATIC_WAVE_PATHS) in msg and "544x544" in msg
    assert r.lib.nr_render_samples_static(r.h, 0, 1) != 0  # sample indices start at 1


def test_static_call_allocates_no_device_memory():
    import torch
    spec = scenes.cornell(res=256, spp=8, depth=8, seed=2)
    sc = capi.Scene(spec)
    warm = capi.Render(sc, tail_max_paths=TAIL_OFF)
    # set-up call (count 0): loads the buffer's module on this device
    assert warm.lib.nr_render_samples_static(warm.h, 1, 0) == 0, last_error()
    assert warm.lib.nr_render_samples_static(warm.h, 1, 2) == 0, last_error()
    fresh = capi.Render(sc, tail_max_paths=TAIL_OFF)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert fresh.lib.nr_render_samples_static(fresh.h, 1, 4) == 0, last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert fresh.layer(0).mean() > 0


def test_static_renders_reference_mode_only():
    spec = scenes.cornell(res=32, spp=3, depth=4, seed=0)
    sc = capi.Scene(spec)
    r = capi.Render(sc, mode=capi.MODE_PERF)
    assert r.lib.nr_render_samples_static(r.h, 1, 1) == NR_ERR_STATE
    assert "NR_MODE_REFERENCE" in last_error()
