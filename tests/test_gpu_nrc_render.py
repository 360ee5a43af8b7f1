"""The radiance cache inside the wavefront (nr_render_set_nrc): paths stop at
their second hit and add the cache's radiance, one path in 16 runs to full
depth and trains the cache after every wave. Judged against an FP64
high-sample perf-mode render: after a short warm-up the cached render has a
clearly lower error than plain perf mode at the same sample count, and its
image mean stays close to the oracle's (the cache's bias is small)."""
import numpy as np
import pytest

from nectarrender_b200 import capi, nrc, scenes

pytestmark = pytest.mark.gpu

ORACLE_SPP = 8192


@pytest.fixture(scope="module")
def cornell():
    spec = scenes.cornell(res=128, spp=ORACLE_SPP + 1, depth=32, seed=0)
    sc = capi.Scene(spec)
    orc = capi.Render(sc, mode=capi.MODE_PERF, fp64_accumulate=1, seed=1000)
    orc.samples(1, ORACLE_SPP)
    return spec, sc, orc.beauty_fp64()


def _rmse(img, oracle):
    # display-referred, like the time-to-error measurement of the benchmark
    d = lambda x: np.sqrt(np.clip(x, 0.0, 1.0))
    return float(np.sqrt(np.mean((d(img) - d(oracle)) ** 2)))


def _cached_render(sc, spec, warm=32):
    lo, hi = sc.bounds()
    cache = nrc.RadianceCache(1 << 18, lo, hi, seed=1)
    r = capi.Render(sc, mode=capi.MODE_PERF, fp64_accumulate=1, seed=spec.seed, samples_per_wave=2)
    r.set_nrc(cache, terminate_bounce=2, train_one_in=16, lr=1e-2, batch=16384, min_steps=8)
    r.samples(ORACLE_SPP // 2, warm)  # warm-up: trains the cache, then discarded
    r.reset()
    return r, cache


def test_cache_lowers_the_error_at_equal_samples(cornell):
    spec, sc, oracle = cornell
    spp = 16
    plain = capi.Render(sc, mode=capi.MODE_PERF, fp64_accumulate=1, seed=spec.seed)
    plain.samples(1, spp)
    e_plain = _rmse(plain.beauty_fp64(), oracle)
    r, cache = _cached_render(sc, spec)
    r.samples(1, spp)
    img = r.beauty_fp64()
    queries, records = r.nrc_stats()
    assert queries > 0 and records > 0
    assert np.isfinite(img).all() and (img >= 0).all()
    e_nrc = _rmse(img, oracle)
    assert e_nrc < 0.8 * e_plain, (e_nrc, e_plain)
    # more samples: still converging, and the mean stays within 5% of the oracle
    r.samples(1 + spp, 48)
    img = r.beauty_fp64()
    assert _rmse(img, oracle) < e_nrc
    assert abs(img.mean() / oracle.mean() - 1.0) < 0.05


def test_detached_cache_gives_the_plain_render(cornell):
    spec, sc, _ = cornell
    r, cache = _cached_render(sc, spec, warm=4)
    r.set_nrc(None)
    r.samples(1, 4)
    plain = capi.Render(sc, mode=capi.MODE_PERF, fp64_accumulate=1, seed=spec.seed, samples_per_wave=2)
    plain.samples(1, 4)
    np.testing.assert_allclose(r.beauty_fp64(), plain.beauty_fp64(), rtol=1e-6, atol=1e-9)


def test_cache_arguments_are_checked(cornell):
    spec, sc, _ = cornell
    lo, hi = sc.bounds()
    cache = nrc.RadianceCache(1 << 12, lo, hi)
    ref = capi.Render(sc, mode=capi.MODE_REFERENCE)
    with pytest.raises(RuntimeError, match="NR_MODE_PERF"):
        ref.set_nrc(cache)
    perf = capi.Render(sc, mode=capi.MODE_PERF)
    with pytest.raises(RuntimeError, match="terminate_bounce"):
        perf.set_nrc(cache, terminate_bounce=spec.ray_depth)
    with pytest.raises(RuntimeError, match="terminate_bounce"):
        perf.set_nrc(cache, terminate_bounce=0)
