"""The depth layer (LayerType DEPTH, one channel, enabled by layer_mask bit
6): the running mean of each sample's first-hit world distance, 0 where the
camera ray leaves the scene. The reference allocates this layer but its
trace_full_kernel never writes it (engine/src/trace.cu:47-79 writes beauty,
diffuse and world normal only); here the wavefront schedule fills it, so the
denoiser can read it. Checked against the per-bounce trace log of the same
sample (bounce 0's world t)."""
import numpy as np
import pytest

from nectarrender_b200 import capi, denoise, scenes

pytestmark = pytest.mark.gpu
NONE = np.uint32(0xFFFFFFFF)


def test_depth_layer_is_the_first_hit_distance():
    spec = scenes.mesh_stress(levels=4, res_h=64, res_w=64, spp=4, depth=6, n_spheres=16,
                              hdri_size=(128, 64), scene_seed=2)
    sc = capi.Scene(spec)
    r = capi.Render(sc, layer_mask=denoise.DENOISE_LAYERS, tail_max_paths=0xFFFFFFFF)
    r.samples(1, 1)
    z = r.layer_channels(6)[0]
    log, _ = capi.Render(sc, tail_max_paths=0xFFFFFFFF).trace_log(1, 1)
    hit = log[:, :, 0].view(np.uint32)[..., 6] != NONE
    want = np.where(hit, log[:, :, 0, 8], 0.0).astype(np.float32)
    np.testing.assert_array_equal(z, want)
    assert hit.any() and (~hit).any()


def test_depth_mean_over_samples_and_default_layers():
    spec = scenes.cornell(res=32, spp=5)
    sc = capi.Scene(spec)
    r = capi.Render(sc, layer_mask=denoise.DENOISE_LAYERS)
    r.samples(1, 4)
    z = r.layer_channels(6)[0]
    assert np.isfinite(z).all() and 1.0 < float(z.mean()) < 3.0   # the box spans 1.5 to 2.5
    with pytest.raises(RuntimeError):
        capi.Render(sc).layer_channels(6)   # not kept by default, as in the reference
