"""Autotuner of the batched propagator (Krylov dimension, tile, budget)."""

import json

import numpy as np
import pytest


def test_budget_meets_the_population_bound():
    from rpm_b200.autotune import budget_for_yield_tolerance
    from rpm_b200.engine import state_error_to_population_bound

    for tol in (1e-6, 1e-4, 3e-3):
        eps = budget_for_yield_tolerance(tol)
        assert state_error_to_population_bound(eps) <= tol * (1 + 1e-12) + eps * eps
        assert eps == pytest.approx(tol / 2)
    with pytest.raises(ValueError):
        budget_for_yield_tolerance(0.0)


def test_krylov_ranges_stay_within_the_batched_limit():
    from rpm_b200.autotune import KRYLOV_EXTENDED, KRYLOV_RANGE

    assert KRYLOV_RANGE == (16, 24, 32, 40)  # the batched benchmark configuration's cap range
    assert set(KRYLOV_RANGE) <= set(KRYLOV_EXTENDED)
    assert min(KRYLOV_EXTENDED) >= 2 and max(KRYLOV_EXTENDED) == 64


@pytest.mark.gpu
def test_tune_picks_a_candidate_and_caches(tmp_path):
    import rpm_b200 as rb
    from rpm_b200 import synthetic
    from rpm_b200.autotune import tune

    full = synthetic.full_system()
    sub = synthetic.prefix_system(full, 5)
    hams = [rb.CompiledFullPairHamiltonian(sub.dimensions, sub.terms(th, ph), left_axes=sub.left_axes,
                                           right_axes=sub.right_axes) for th, ph in synthetic.fibonacci_sphere(2)]
    states = synthetic.random_phase_vectors(sub.dimensions, 8, 11)
    idx = np.array([k % 2 for k in range(8)], dtype=np.int32)
    cache = tmp_path / "tune.json"
    res = tune(hams, list(states), idx, horizon_us=0.05, krylov_dimensions=(16, 24), tiles=(4, 8), cache=cache)
    assert res.krylov_dimension in (16, 24) and res.tile in (4, 8)
    assert res.state_error_budget == pytest.approx(5e-7)
    assert len([t for t in res.trials if "throughput" in t]) == 4
    assert res.throughput == max(t["throughput"] for t in res.trials if "throughput" in t)
    stored = json.loads(cache.read_text())
    assert len(stored) == 1
    again = tune(hams, list(states), idx, horizon_us=0.05, krylov_dimensions=(16, 24), tiles=(4, 8), cache=cache)
    assert again.krylov_dimension == res.krylov_dimension and again.trials == res.trials
    # the tuned propagator reproduces the FP64 path within the yield tolerance
    times = np.arange(201) * 0.00125
    out = res.propagator(hams).propagate(list(states[:2]), times, system_index=[0, 1], lifetime_us=1.0)
    for b in range(2):
        ref = rb.AdaptiveLanczosPropagator(hams[b], minimum_dimension=8, maximum_dimension=40,
                                           state_error_budget=1e-10).propagate(
            states[b], times, rb.SingletPopulationObservable(sub.dimensions))
        assert abs(out.yields[b] - rb.integrate_yield(times, ref.observable_values, 1.0)) < 1e-6
