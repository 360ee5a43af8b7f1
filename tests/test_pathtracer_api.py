"""The `_pathtracer` module mirrors the reference's Python API."""
import pytest

import nectarrender_b200 as nb
from nectarrender_b200 import scenes


@pytest.fixture(scope="module")
def pt():
    return nb.pathtracer()


def test_submodules_and_names(pt):
    for path in ["core.vector.Vector3", "core.vector.Color", "core.vector.Vector2",
                 "material.Material", "material.texture.Texture", "hittable.Hittable",
                 "light.Skylight", "scene.Scene", "engine.RenderEngine",
                 "engine.camera.Camera", "engine.camera.CameraParams", "data.LayerType",
                 "data.StreamConfig", "data.TonemapMethod", "data.DataObject", "cuda.destroy_cublas_handle"]:
        obj = pt
        for part in path.split("."):
            obj = getattr(obj, part)
        assert obj is not None, path


def test_factories(pt):
    V3, C = pt.core.vector.Vector3, pt.core.vector.Color
    M, H = pt.material.Material, pt.hittable.Hittable
    m = M.lambertian(C(0.5, 0.5, 0.5))
    assert repr(m) == "Material(type = Lambertian)"
    q = H.quad(V3(0.0, 0.0, 0.0), V3(0.0, 90.0, 0.0), V3(1.0), m)
    light = H.object_light(q, 15.0, C(1.0, 1.0, 1.0))
    assert light.is_light() and not q.is_light()
    with pytest.raises(RuntimeError):
        H.object_light(light, 1.0, C(1.0, 1.0, 1.0))
    with pytest.raises(RuntimeError, match="Failed to load OBJ"):
        H.mesh("/nonexistent.obj")
    sky = pt.light.Skylight.simple()
    sky.config_simple().start = C(0.1, 0.2, 0.3)
    assert sky.config_simple().start.r() == pytest.approx(0.1)
    assert M.pbr().texture_count() == 5


def test_scene_and_engine_surface(pt):
    spec = scenes.cornell(res=16, spp=2)
    scene, cam, keep = scenes.to_pathtracer(spec, pt)
    eng = pt.engine.RenderEngine(cam, 8, 0)
    assert eng.n_samples() == 3 and eng.max_depth() == 8
    layers = eng.layers()
    assert layers.beauty.is_enabled() and not layers.depth.is_enabled()
    assert layers.beauty.shape() == [3, 16, 16]
    with pytest.raises(RuntimeError, match="before set_scene"):
        eng.render()
    if nb.device_count() == 0:
        with pytest.raises(RuntimeError, match="no CUDA device"):
            eng.set_scene(scene)


@pytest.mark.parametrize("mode", ["RGB", "RGBA"])
def test_image_texture_planes_match_the_reference_loader(pt, tmp_path, mode):
    """Texture.from_image builds its planes as the reference's loader does
    (texture.h:8-26): right for RGB, and for RGBA with the reference's
    i * 3 + c indexing of four-channel pixels."""
    import numpy as np
    import oracle
    Image = pytest.importorskip("PIL.Image")
    if not oracle.REF_CPU_SO.exists():
        pytest.skip("reference host build not present")
    rng = np.random.default_rng(5)
    nch = len(mode)
    px = rng.integers(0, 256, (5, 7, nch), dtype=np.uint8)
    path = tmp_path / f"t_{mode}.png"
    Image.fromarray(px, mode).save(path)
    ours = pt.material.texture.Texture.from_image(str(path), 0.5)
    ref = oracle.RefCPU().load_image_uint8(str(path))
    assert (ours.C, ours.H, ours.W) == ref.shape == (nch, 5, 7)
    assert np.array_equal(ours.texels, ref)
    if mode == "RGB":   # planes are the image's channels
        assert np.array_equal(ref, px.transpose(2, 0, 1))
    else:               # the reference's four-channel quirk: shifted planes
        assert not np.array_equal(ref[:3], px[..., :3].transpose(2, 0, 1))
