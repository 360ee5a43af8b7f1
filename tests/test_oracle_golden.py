"""The CPU oracle against fixtures produced by the reference's own
integrator (tests/golden/make_golden.py) and, where the reference build is
present, against that build live. Comparisons are bit-exact: the oracle
restates the reference's arithmetic in the same order."""
import numpy as np
import pytest

import oracle
from nectarrender_b200 import scenes
from tests.golden.make_golden import HERE as GOLDEN, cornell_spec, local_mesh_spec

pytestmark = []


@pytest.fixture(scope="module")
def orc():
    return oracle.Oracle()


def test_philox_matches_curand_fixture(orc):
    g = np.load(GOLDEN / "cornell24.npz")
    assert np.array_equal(orc.uniforms(0, 5, 64), g["philox_0_5"])
    assert np.array_equal(orc.uniforms(54321, 1000, 64), g["philox_54321_1000"])


def test_n_rooks_host_order(orc):
    g = np.load(GOLDEN / "cornell24.npz")
    assert np.array_equal(orc.n_rooks(4, 0, draw_rtl=1), g["n_rooks_4_0"])
    # the other argument order gives a different pattern
    assert not np.array_equal(orc.n_rooks(4, 0, draw_rtl=0), g["n_rooks_4_0"])


@pytest.mark.parametrize("s", [1, 2])
def test_cornell_raw_samples(orc, s):
    g = np.load(GOLDEN / "cornell24.npz")
    b, d, n, p, _ = orc.render(cornell_spec(), s, mode=0, draw_rtl=1)
    assert np.array_equal(b, g[f"s{s}_beauty"])
    assert np.array_equal(d, g[f"s{s}_diffuse"])
    assert np.array_equal(n, g[f"s{s}_normal"])
    assert np.array_equal(p, g[f"s{s}_primary"])


def test_cornell_running_mean_and_fp64(orc):
    g = np.load(GOLDEN / "cornell24.npz")
    b, d, n, _, b64 = orc.render(cornell_spec(), 1, count=3, mode=1, draw_rtl=1, fp64=True)
    assert np.array_equal(b, g["acc_beauty"])
    assert np.array_equal(d, g["acc_diffuse"])
    assert np.array_equal(n, g["acc_normal"])
    assert np.array_equal(b64, g["acc_beauty64"])


def test_mesh_scene_readers_and_samples(orc):
    g = np.load(GOLDEN / "mesh_small.npz")
    spec = local_mesh_spec()
    P, N, T, UV, tris = orc.load_obj(spec.meshes[0])
    for a, k in zip((P, N, T, UV, tris), ("obj_P", "obj_N", "obj_T", "obj_UV", "obj_tris")):
        assert np.array_equal(a, g[k]), k
    assert np.array_equal(orc.load_hdr(spec.sky["path"]), g["hdr"])
    b, d, n, p, _ = orc.render(spec, 1, mode=0, draw_rtl=1)
    assert np.array_equal(b, g["s1_beauty"])
    assert np.array_equal(d, g["s1_diffuse"])
    assert np.array_equal(n, g["s1_normal"])
    assert np.array_equal(p, g["s1_primary"])
    b, d, n, _, b64 = orc.render(spec, 1, count=2, mode=1, draw_rtl=1, fp64=True)
    assert np.array_equal(b, g["acc_beauty"])
    assert np.array_equal(b64, g["acc_beauty64"])
    sah, nodes = orc.mesh_sah(spec)
    assert sah == g["sah"][0] and nodes == g["sah_nodes"][0]


@pytest.mark.skipif(not oracle.REF_CPU_SO.exists(), reason="reference host build not present")
@pytest.mark.parametrize("seed", [3, 11])
def test_oracle_matches_reference_live(orc, seed):
    """Fresh seeds, edge material mix and a medium, against the reference build."""
    ref = oracle.RefCPU()
    spec = scenes.mesh_stress(levels=2, res_h=16, res_w=16, spp=3, depth=16, n_spheres=12,
                              hdri_size=(64, 32), scene_seed=seed)
    # wrap a cube medium around the mesh (the participating-medium configuration)
    spec.objects.append(scenes.obj(scenes.MEDIUM, scenes.isotropic((0.9, 0.9, 0.9)),
                                   (0, 0, 0), (0, 20, 0), (2, 2, 2), wrapped=scenes.CUBE,
                                   density=0.5))
    for s in (1, 2):
        a = orc.render(spec, s, mode=0, draw_rtl=1)
        b = ref.render(spec, s, mode=0)
        for k in range(4):
            assert np.array_equal(a[k], b[k]), (s, k)


@pytest.mark.skipif(not oracle.REF_CPU_SO.exists(), reason="reference host build not present")
def test_oracle_matches_reference_defocus_and_rotated_cubes(orc):
    """Thin-lens defocus and rotated cubes of three materials, against the
    reference build, bit for bit."""
    ref = oracle.RefCPU()
    spec = scenes.cornell_cubes(res=16, spp=3)
    for s in (1, 2):
        a = orc.render(spec, s, mode=0, draw_rtl=1)
        b = ref.render(spec, s, mode=0)
        for k in range(4):
            assert np.array_equal(a[k], b[k]), (s, k)
    assert a[0].any()


@pytest.mark.skipif(not oracle.REF_CPU_SO.exists(), reason="reference host build not present")
@pytest.mark.parametrize("make", [scenes.cornell_textured, scenes.cornell_textured_mesh])
def test_oracle_matches_reference_image_textures(orc, make):
    """Image textures (wrapped checker albedo, PBR albedo, roughness,
    metallic and normal maps on a sphere, a rotated cube and a uv-mapped
    mesh read from an OBJ with texture coordinates), against the reference
    build, bit for bit."""
    ref = oracle.RefCPU()
    spec = make(res=16, spp=3)
    for s in (1, 2):
        a = orc.render(spec, s, mode=0, draw_rtl=1)
        b = ref.render(spec, s, mode=0)
        for k in range(4):
            assert np.array_equal(a[k], b[k]), (s, k)
    # the textures are seen: the diffuse layer differs from the untextured box
    plain = orc.render(scenes.cornell(res=16, spp=3), 1, mode=0, draw_rtl=1)
    assert (a[1] != plain[1]).mean() > 0.2


def test_empty_rows_request(orc):
    b, *_ = orc.render(cornell_spec(), 1, mode=0, rows=(5, 5))
    assert not b.any()
