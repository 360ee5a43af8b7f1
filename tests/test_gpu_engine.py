"""The reference's Python API (`_pathtracer`) end to end on the GPU."""
import ctypes

import numpy as np
import pytest

import nectarrender_b200 as nb
from nectarrender_b200 import capi, scenes

pytestmark = pytest.mark.gpu


def test_render_engine_matches_c_abi():
    pt = nb.pathtracer()
    spec = scenes.cornell(res=32, spp=4)
    scene, cam, keep = scenes.to_pathtracer(spec, pt)
    eng = pt.engine.RenderEngine(cam, spec.ray_depth, spec.seed)
    eng.set_scene(scene)
    frames = []
    eng.on_frame_finished = lambda i: frames.append(i)
    eng.render()
    assert frames == [2, 3, 4, 5]                     # one hook per sample, after each
    beauty = eng.layers().beauty
    ptr = beauty.device_ptr()
    assert ptr != 0 and beauty.shape() == [3, 32, 32]
    # the same scene through the C ABI gives the same running mean
    sc = capi.Scene(spec)
    r = capi.Render(sc)
    r.render_all()
    ref = r.layer(0)
    u8 = beauty.numpy()
    expect = np.clip(np.nan_to_num(ref), 0, 1) * 255.0
    assert np.abs(u8.astype(np.float64) - expect.astype(np.uint8)).max() <= 1
    st = eng.stream()
    cfg = pt.data.StreamConfig()
    st.update_config(cfg)
    p = st.readback()
    arr = np.ctypeslib.as_array((ctypes.c_uint8 * (3 * 32 * 32)).from_address(p)).reshape(3, 32, 32)
    assert arr.max() > 0


def test_engine_restart_and_stop_requests():
    pt = nb.pathtracer()
    spec = scenes.cornell(res=16, spp=6)
    scene, cam, keep = scenes.to_pathtracer(spec, pt)
    eng = pt.engine.RenderEngine(cam, 8, 0)
    eng.set_scene(scene)
    seen = []

    def hook(i):
        seen.append(i)
        if i == 3:
            eng.requests().stop()
    eng.on_frame_finished = hook
    eng.poll_updates = lambda: pt.engine.EnginePollResponse()
    rc = eng.render()
    assert rc == 1 and seen == [2, 3]      # stopped before the third sample
