"""Per-sample parity of the CUDA integrator (called through the C ABI) with
the CPU oracle and with the reference's own CUDA build, plus the display
transform. Tolerance: per-sample radiance within 1e-4 relative; a sample
whose path takes a different branch after a rounding difference (fast-math
device math versus host libm, or a different closest hit at an exact tie)
differs wholesale, so the bar is a fraction of values, stated per test."""
import numpy as np
import pytest

import oracle
from nectarrender_b200 import capi, scenes
from tests.gpu_util import frac_close

pytestmark = pytest.mark.gpu
RTL = 0  # the reference's CUDA build draws multi-draw arguments left to right


@pytest.fixture(scope="module")
def orc():
    return oracle.Oracle()


@pytest.fixture(scope="module")
def refcuda():
    if not oracle.REF_CUDA_SO.exists():
        pytest.skip("reference CUDA build not present")
    return oracle.RefCUDA()


def test_reference_cuda_draw_order(refcuda):
    assert refcuda.probe_draw_order() == (0, 0)
    assert capi.device_draw_order() == 0


@pytest.fixture(scope="module")
def cornell():
    spec = scenes.cornell(res=64, spp=8)
    sc = capi.Scene(spec)
    return spec, sc, capi.Render(sc)


@pytest.mark.parametrize("s", [1, 2, 5])
def test_cornell_samples_vs_oracle(cornell, orc, s):
    spec, _, r = cornell
    b, d, n, p = r.sample_layers(s)
    ob, od, on, op, _ = orc.render(spec, s, mode=0, draw_rtl=RTL)
    assert frac_close(b, ob) >= 0.99
    assert frac_close(d, od) >= 0.99
    assert frac_close(n, on) >= 0.99
    assert (p == op).mean() >= 0.999   # primary-hit object/triangle ids


@pytest.mark.parametrize("s", [1, 3])
def test_cornell_samples_vs_reference_cuda(cornell, refcuda, s):
    spec, _, r = cornell
    b, d, n, _ = r.sample_layers(s)
    rb, rd, rn, _ = refcuda.render(spec, s, mode=0)
    assert frac_close(b, rb) >= 0.995
    assert frac_close(d, rd) >= 0.995
    assert frac_close(n, rn) >= 0.999


def test_cornell_running_mean_vs_reference_cuda(cornell, refcuda):
    spec, _, r = cornell
    r.reset()
    r.render_all()
    acc = r.layer(0)
    rb, *_ = refcuda.render(spec, 1, count=spec.camera["samples_per_pixel"] - 1, mode=1)
    assert frac_close(acc, rb) >= 0.99
    assert abs(acc.mean() - rb.mean()) <= 1e-3 * rb.mean()


@pytest.fixture(scope="module")
def mesh_scene():
    spec = scenes.mesh_stress(levels=5, res_h=64, res_w=64, spp=4, depth=12, n_spheres=32,
                              hdri_size=(256, 128), scene_seed=1)
    sc = capi.Scene(spec)
    return spec, sc, capi.Render(sc)


@pytest.mark.parametrize("s", [1, 2])
def test_mesh_hdri_samples(mesh_scene, orc, refcuda, s):
    spec, _, r = mesh_scene
    b, d, n, p = r.sample_layers(s)
    rb, rd, rn, _ = refcuda.render(spec, s, mode=0)
    assert frac_close(b, rb) >= 0.99
    assert frac_close(n, rn) >= 0.999
    *_, op, _ = orc.render(spec, s, mode=0, draw_rtl=RTL)
    hit = op != 0xFFFFFFFF
    assert hit.any()
    assert (p == op).mean() >= 0.999


@pytest.mark.parametrize("variant,mesh_leaf,tlas_leaf,spw,schedule", [
    (4, 3, 1, 0, capi.SCHEDULE_WAVEFRONT),
    (1004, 1, 1, 0, capi.SCHEDULE_WAVEFRONT),   # 128-register shading kernel, tail off
    (6, 1, 2, 1, capi.SCHEDULE_WAVEFRONT),
    (8, 2, 3, 3, capi.SCHEDULE_WAVEFRONT),
    (5, 1, 1, 0, capi.SCHEDULE_MEGAKERNEL),
    (14, 1, 1, 0, capi.SCHEDULE_WAVEFRONT),
    (15, 3, 2, 2, capi.SCHEDULE_WAVEFRONT),
    (16, 2, 1, 0, capi.SCHEDULE_WAVEFRONT),
    (515, 1, 1, 0, capi.SCHEDULE_WAVEFRONT),
    (514, 1, 1, 0, capi.SCHEDULE_WAVEFRONT),    # the flattened traversal without the vote
    (84, 2, 1, 2, capi.SCHEDULE_WAVEFRONT),
])
def test_tuning_knobs_do_not_change_samples(mesh_scene, refcuda, variant, mesh_leaf, tlas_leaf,
                                            spw, schedule):
    """Every traversal variant, leaf size, wave size and schedule the tuner
    may pick renders the same per-sample images."""
    spec, _, _ = mesh_scene
    sc = capi.Scene(spec, mesh_leaf=mesh_leaf, tlas_leaf=tlas_leaf)
    extra = {}
    if variant >= 1000:  # other shading kernel and no tail hand-off
        variant, extra = variant - 1000, {"shade_variant": 4, "tail_max_paths": 0xFFFFFFFF}
    r = capi.Render(sc, extend_variant=variant, samples_per_wave=spw, schedule=schedule, **extra)
    r.samples(1, 3)
    acc = r.layer(0)
    rb, *_ = refcuda.render(spec, 1, count=3, mode=1)
    assert frac_close(acc, rb) >= 0.99
    b, d, n, p = r.sample_layers(2)
    rb2, _, rn2, _ = refcuda.render(spec, 2, mode=0)
    assert frac_close(b, rb2) >= 0.99
    assert frac_close(n, rn2) >= 0.999


@pytest.mark.parametrize("mode", [capi.MODE_REFERENCE, capi.MODE_PERF])
def test_material_sorted_shading_gives_the_same_images(mesh_scene, mode):
    """Shading each bounce's queue grouped by material type changes only the
    order in which paths are shaded: every path draws from its own random
    stream and owns its accumulator, so the images are bit-identical."""
    spec, sc, _ = mesh_scene
    a = capi.Render(sc, mode=mode, sort_materials=1)
    b = capi.Render(sc, mode=mode, sort_materials=-1)
    a.samples(1, 3)
    b.samples(1, 3)
    for layer in (0, 1, 4):
        np.testing.assert_array_equal(a.layer(layer), b.layer(layer))


def test_wave_graphs_replay_the_same_samples(mesh_scene):
    """Waves replayed from captured CUDA graphs read their first sample index
    from device memory; three calls in a row (direct, capture, replay) equal
    direct launches."""
    spec, sc, _ = mesh_scene
    g = capi.Render(sc, samples_per_wave=1)
    d = capi.Render(sc, samples_per_wave=1, use_graphs=0)
    for first in (1, 2, 3):
        g.samples(first, 1)
        d.samples(first, 1)
        for layer in (0, 1, 4):
            np.testing.assert_array_equal(g.layer(layer), d.layer(layer))
    captured, replays = g.graph_stats()
    assert captured == 1 and replays == 2
    assert d.graph_stats() == (0, 0)


def test_participating_medium_samples(orc, refcuda):
    spec = scenes.mesh_stress(levels=3, res_h=48, res_w=48, spp=2, depth=32, n_spheres=8,
                              hdri_size=(128, 64), scene_seed=2)
    spec.objects.append(scenes.obj(scenes.MEDIUM, scenes.isotropic((0.9, 0.9, 0.9)), (0, 0, 0),
                                   (0, 0, 0), (2, 2, 2), wrapped=scenes.CUBE, density=0.5))
    sc = capi.Scene(spec)
    r = capi.Render(sc)
    b, *_ = r.sample_layers(1)
    rb, *_ = refcuda.render(spec, 1, mode=0)
    assert np.isfinite(b).all()
    assert frac_close(b, rb) >= 0.98


@pytest.mark.parametrize("s", [1, 2])
def test_defocus_and_rotated_cubes(orc, refcuda, s):
    """Thin-lens defocus and rotated cubes (Lambertian, rough metal, glass)
    per sample, against the oracle and the reference's CUDA build."""
    spec = scenes.cornell_cubes(res=64, spp=3)
    r = capi.Render(capi.Scene(spec))
    b, d, n, p = r.sample_layers(s)
    ob, od, on, op, _ = orc.render(spec, s, mode=0, draw_rtl=RTL)
    assert frac_close(b, ob) >= 0.99
    assert frac_close(n, on) >= 0.99
    assert (p == op).mean() >= 0.999
    rb, rd, rn, _ = refcuda.render(spec, s, mode=0)
    assert frac_close(b, rb) >= 0.99
    assert frac_close(d, rd) >= 0.99
    assert frac_close(n, rn) >= 0.999


@pytest.mark.parametrize("make", [scenes.cornell_textured, scenes.cornell_textured_mesh])
@pytest.mark.parametrize("s", [1, 2])
def test_image_textures_and_normal_maps(orc, refcuda, s, make):
    """Image textures and normal maps per sample (on analytic shapes, and on
    a uv-mapped OBJ mesh), against the oracle and the reference's CUDA build
    (its Texture set up from the same bytes)."""
    spec = make(res=64, spp=3)
    r = capi.Render(capi.Scene(spec))
    b, d, n, p = r.sample_layers(s)
    ob, od, on, op, _ = orc.render(spec, s, mode=0, draw_rtl=RTL)
    assert frac_close(b, ob) >= 0.99
    assert frac_close(d, od) >= 0.999
    assert (p == op).mean() >= 0.999
    rb, rd, rn, _ = refcuda.render(spec, s, mode=0)
    assert frac_close(b, rb) >= 0.99
    assert frac_close(d, rd) >= 0.999
    assert frac_close(n, rn) >= 0.999


def test_edge_sizes_not_multiple_of_tiles(orc):
    spec = scenes.cornell(res=37, spp=2)
    spec.camera["resolution"] = (37.0, 37.0)
    sc = capi.Scene(spec)
    r = capi.Render(sc)
    b, d, n, p = r.sample_layers(1)
    ob, *_ = orc.render(spec, 1, mode=0, draw_rtl=RTL)
    assert b.shape == (3, 37, 37)
    assert frac_close(b, ob) >= 0.99


@pytest.mark.parametrize("cfg", [
    dict(gamma=True, white_balance=False, tonemap=True, method=0),
    dict(gamma=True, white_balance=True, tonemap=True, method=0, temperature=5200.0, tint=12.0),
    dict(gamma=True, white_balance=True, tonemap=True, method=2, temperature=9000.0),
    dict(gamma=False, white_balance=False, tonemap=True, method=1, white_point=2.0, alpha=0.7),
])
def test_display_transform(cornell, cfg):
    spec, _, r = cornell
    r.reset()
    r.samples(1, 4)
    img = r.layer(0)
    c = capi.stream_config(**cfg)
    f = r.display_float(0, c)
    u8 = r.readback(0, c)
    o8, of = oracle.display(img, c)
    assert np.abs(f - of).max() <= 5e-5
    assert (np.abs(u8.astype(int) - o8.astype(int)) > 1).sum() == 0
    assert (u8 != o8).mean() <= 0.005


def test_fp64_accumulator(cornell):
    spec, sc, _ = cornell
    r = capi.Render(sc, fp64_accumulate=1)
    r.samples(1, 6)
    acc = r.layer(0)
    acc64 = r.beauty_fp64()
    assert np.allclose(acc, acc64, rtol=1e-4, atol=1e-6)
