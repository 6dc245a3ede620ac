"""Autotuner of the batched propagator (Krylov dimension, tile, reorthogonalisation, budget)."""

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
    res = tune(hams, list(states), idx, horizon_us=0.05, krylov_dimensions=(16, 24), tiles=(4, 8),
               reorth_periods=(0, 6), cache=cache)
    assert res.krylov_dimension in (16, 24) and res.tile in (4, 8) and res.reorth_period in (0, 6)
    assert res.state_error_budget == pytest.approx(5e-7)
    measured = [t for t in res.trials if "throughput" in t]
    assert len(measured) == 8
    assert all(t["yield_err_prefix"] is not None for t in measured)
    assert res.throughput == max(t["throughput"] for t in measured if t["accepted"])
    stored = json.loads(cache.read_text())
    assert len(stored) == 1
    again = tune(hams, list(states), idx, horizon_us=0.05, krylov_dimensions=(16, 24), tiles=(4, 8),
                 reorth_periods=(0, 6), cache=cache)
    assert again.krylov_dimension == res.krylov_dimension and again.trials == res.trials
    # the tuned propagator reproduces the FP64 path within the yield tolerance
    times = np.arange(201) * 0.00125
    out = res.propagator(hams).propagate(list(states[:2]), times, system_index=[0, 1], lifetime_us=1.0)
    for b in range(2):
        ref = rb.AdaptiveLanczosPropagator(hams[b], minimum_dimension=8, maximum_dimension=40,
                                           state_error_budget=1e-10).propagate(
            states[b], times, rb.SingletPopulationObservable(sub.dimensions))
        assert abs(out.yields[b] - rb.integrate_yield(times, ref.observable_values, 1.0)) < 1e-6


def test_spread_selection_takes_every_shape_in_turn():
    from rpm_b200.autotune import spread_selection

    shape_of = ["a", "a", "b", "c"]          # systems 0, 1 share a shape
    sample = [0, 1, 0, 1, 0, 2, 2, 3, 3, 3]  # system of each sample trajectory
    sel = spread_selection(sample, shape_of, 3)
    assert [shape_of[sample[p]] for p in sel] == ["a", "b", "c"]
    sel = spread_selection(sample, shape_of, 7)
    got = [shape_of[sample[p]] for p in sel]
    assert got.count("a") == 3 and got.count("b") == 2 and got.count("c") == 2
    assert list(sel) == sorted(sel)
    assert len(spread_selection(sample, shape_of, 50)) == len(sample)
