"""The autotuner's cost model on the host (no GPU): method and leaf-level
choices from fixed kernel rates and the library's exact interaction tables,
and the rate cache's round trip."""
import json

import pytest

SIGMA = 0.002
KS = 2 * SIGMA * SIGMA
BOX = (0.0, 1.0, 0.0, 1.0)


@pytest.fixture
def tuner():
    from pfblob.tune import DEFAULT_RATES, Tuner
    return Tuner(rates=dict(DEFAULT_RATES))


def test_small_sets_and_exact_tolerance_use_the_direct_sum(tuner):
    assert tuner.choose(50, KS, BOX) == (1, 0)
    assert tuner.choose(1000, KS, BOX) == (1, 0)
    assert tuner.choose(1 << 20, KS, BOX, tol=0.0) == (1, 0)


def test_large_sets_use_the_fmm_with_growing_leaf_level(tuner):
    levels = []
    for n in (1 << 15, 1 << 16, 1 << 18, 1 << 20, 1 << 22):
        method, level = tuner.choose(n, KS, BOX)
        assert method == 0 and 3 <= level <= 11, (n, method, level)
        levels.append(level)
    assert levels == sorted(levels)
    assert levels[-1] > levels[0]


def test_choice_minimises_the_model(tuner):
    """The chosen leaf level is the cheapest of the levels the model tries,
    and cheaper than the direct sum."""
    n = 1 << 20
    method, level = tuner.choose(n, KS, BOX)
    from pfblob.induced import default_cutoff
    cut = default_cutoff(KS, 1e-6)
    best = tuner.fmm_cost(n, level, 1.0, cut)
    for other in range(max(3, level - 2), level + 3):
        assert best <= tuner.fmm_cost(n, other, 1.0, cut) * (1 + 1e-12)
    assert best < float(n) * n / tuner.rates["r_direct"]


def test_batched_sets_switch_to_the_fmm_no_later(tuner):
    """Inside a captured batch the FMM's per-call latency overlaps other work,
    so the direct-to-FMM crossover comes at the same or a smaller size."""
    def crossover(batch):
        for k in range(8, 24):
            if tuner.choose(1 << k, KS, BOX, batch=batch)[0] == 0:
                return k
        return None
    plain, batched = crossover(False), crossover(True)
    assert plain is not None and batched is not None and batched <= plain


def test_box_scaling_is_invariant(tuner):
    """The model depends on the cutoff relative to the box: scaling blobs,
    box and sigma together leaves the choice unchanged."""
    for s in (1e-3, 1.0, 250.0):
        ks = 2 * (SIGMA * s) ** 2
        assert tuner.choose(1 << 18, ks, tuple(v * s for v in BOX)) == tuner.choose(1 << 18, KS, BOX)


def test_rate_cache_round_trip(tmp_path, monkeypatch):
    from pfblob.tune import CACHE_ENV, DEFAULT_RATES, Tuner
    path = tmp_path / "rates.json"
    monkeypatch.setenv(CACHE_ENV, str(path))
    t = Tuner(rates=dict(DEFAULT_RATES, r_p2p=1.23e12))
    t.save()
    assert json.loads(path.read_text())["r_p2p"] == 1.23e12
    assert Tuner().rates["r_p2p"] == 1.23e12
    path.write_text("not json")
    assert Tuner().rates["r_p2p"] == DEFAULT_RATES["r_p2p"]  # unreadable cache: defaults
