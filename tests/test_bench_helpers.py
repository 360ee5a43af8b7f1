"""Host-side helpers of bench.py (no GPU): the time-at-error interpolation of
the time-to-RMSE curves, the section guard, the oracle statistics and the
sample-index slices of the ranks."""
import bench


def test_time_at_interpolates_in_log_log():
    curve = [[1, 10.0, 0.4, 0.39], [2, 20.0, 0.1, 0.09], [4, 40.0, 0.05, 0.04]]
    assert bench._time_at(curve, 0.4) == 10.0
    t = bench._time_at(curve, 0.2)
    assert 10.0 < t < 20.0 and abs(t - 10.0 * 2 ** 0.5) < 1e-9   # halfway in log error
    assert bench._time_at(curve, 0.01) is None
    assert bench._time_at([[1, 5.0, 0.001]], 0.01) == 5.0


def test_section_records_failures():
    def boom():
        raise ValueError("x")
    assert bench.section(False, boom) is None
    assert "ValueError" in bench.section(True, boom)["error"]
    assert bench.section(True, lambda a: a + 1, 1) == 2


def test_oracle_stats():
    import numpy as np
    rng = np.random.default_rng(0)
    truth = rng.uniform(0.1, 0.5, (3, 32, 32))
    h0 = truth + rng.normal(0, 0.01, truth.shape)
    h1 = truth + rng.normal(0, 0.01, truth.shape)
    between, err, share = bench.oracle_stats(h0, h1)
    assert between > 0 and err == 0.5 * between
    assert 0.0 < share["top_0.1pct_pixels"] <= share["top_1pct_pixels"] <= 1.0
    mean = 0.5 * (h0 + h1)
    d = lambda x: np.sqrt(np.clip(x, 0, 1))
    true_err = float(np.sqrt(np.mean((d(mean) - d(truth)) ** 2)))
    assert 0.5 * err < true_err < 2.0 * err


def test_sample_slices_stay_in_the_32_bit_streams():
    import pytest
    h, w, S = 1080, 1920, 4
    cap = bench.sample_cap(h, w)
    assert w * h * (cap + 1) <= 0xFFFFFFFF < w * h * (cap + 2)
    for world in (1, 2, 4, 8):
        for steps in (5, 64, 300):
            spp = min(cap, max(256, S * steps * world)) + 1
            for step in range(steps):
                firsts = [bench.sample_first(step, r, world, S, spp) for r in range(world)]
                assert len(set(firsts)) == world                     # disjoint within a step
                assert min(firsts) >= 1 and max(firsts) + S <= spp   # inside the camera's range
    # no wrap while the run fits: every slice once
    seen = {bench.sample_first(k, r, 2, S, 2 * S * 10 + 1) for k in range(10) for r in range(2)}
    assert len(seen) == 20
    with pytest.raises(ValueError):
        bench.sample_first(0, 0, 8, S, 8)
