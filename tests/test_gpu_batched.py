"""Batched mixed-precision path against the FP64 plain path (GPU).

Bar (the batched path's contract): singlet yield within 1e-6 of the FP64
path for every trajectory; populations within 1e-5 at every time.
"""

import math

import numpy as np
import pytest

from conftest import terms_from

pytestmark = pytest.mark.gpu

YIELD_TOL = 1e-6
POP_TOL = 1e-5


@pytest.fixture(scope="module")
def rb():
    import rpm_b200

    return rpm_b200


def _plain(rb, h, psi, times, knobs):
    res = rb.AdaptiveLanczosPropagator(h, **knobs).propagate(psi, times, rb.SingletPopulationObservable(h.dimensions))
    return res.observable_values


def test_small_system_batch_matches_fp64(rb, golden):
    from rpm_b200.batched import BatchedPropagator

    dims = tuple(int(v) for v in golden["small_dims"])
    h = rb.CompiledFullPairHamiltonian(dims, terms_from(golden, "small", rb.LocalTerm),
                                       left_axes=tuple(golden["small_left"]), right_axes=tuple(golden["small_right"]))
    times = golden["small_times"]
    psi = golden["small_psi0"]
    bp = BatchedPropagator([h], krylov_dimension=30, state_error_budget=1e-9)
    out = bp.propagate(psi, times, lifetime_us=1.0)
    for b in range(len(psi)):
        ref = _plain(rb, h, psi[b], times, dict(minimum_dimension=30, maximum_dimension=30, state_error_budget=1e-10))
        assert np.max(np.abs(out.observable_values[b] - ref)) < POP_TOL
        y_ref = rb.integrate_yield(times, ref, 1.0)
        assert abs(out.yields[b] - y_ref) < YIELD_TOL
    assert all(s.accepted_steps > 0 and s.rejected_steps == 0 for s in out.stats)


def test_orientations_and_uneven_sizes_in_one_batch(rb):
    from rpm_b200 import synthetic
    from rpm_b200.batched import BatchedPropagator

    full = synthetic.full_system()
    systems, hams = [], []
    for per, (th, ph) in ((3, (0.3, 0.0)), (3, (1.2, 2.0)), (5, (0.7, 1.1))):
        sub = synthetic.prefix_system(full, per)
        systems.append(sub)
        hams.append(rb.CompiledFullPairHamiltonian(sub.dimensions, sub.terms(th, ph), left_axes=sub.left_axes,
                                                   right_axes=sub.right_axes))
    idx = [0, 1, 2, 0, 2]
    psi = [synthetic.random_phase_vectors(systems[k].dimensions, 1, 100 + b)[0] for b, k in enumerate(idx)]
    times = np.arange(161) * 0.00125
    bp = BatchedPropagator(hams, krylov_dimension=32, state_error_budget=1e-9)
    out = bp.propagate(psi, times, system_index=idx, lifetime_us=1.0, return_final_states=True)
    for b, k in enumerate(idx):
        ref = _plain(rb, hams[k], psi[b], times, dict(minimum_dimension=8, maximum_dimension=40,
                                                      state_error_budget=1e-10))
        assert np.max(np.abs(out.observable_values[b] - ref)) < POP_TOL
        assert abs(out.yields[b] - rb.integrate_yield(times, ref, 1.0)) < YIELD_TOL
        n = hams[k].dimension
        norm = float(out.final_states[b, :n].abs().pow(2).sum().sqrt())
        assert abs(norm - 1.0) < 1e-5


def test_full_size_short_horizon(rb):
    from rpm_b200 import synthetic
    from rpm_b200.batched import BatchedPropagator

    full = synthetic.full_system()
    h = rb.CompiledFullPairHamiltonian(full.dimensions, full.terms(math.pi / 4, 0.0), left_axes=full.left_axes,
                                       right_axes=full.right_axes)
    psi = synthetic.random_phase_vectors(full.dimensions, 2, 7)
    times = np.arange(41) * 0.00125
    out = BatchedPropagator([h], krylov_dimension=32, state_error_budget=1e-8).propagate(psi, times, lifetime_us=1.0)
    for b in range(2):
        ref = _plain(rb, h, psi[b], times, dict(minimum_dimension=8, maximum_dimension=40, state_error_budget=1e-10))
        assert np.max(np.abs(out.observable_values[b] - ref)) < POP_TOL
        assert abs(out.yields[b] - rb.integrate_yield(times, ref, 1.0)) < YIELD_TOL


def test_batched_rejects_bad_times(rb, golden):
    from rpm_b200.batched import BatchedPropagator

    dims = tuple(int(v) for v in golden["small_dims"])
    h = rb.CompiledFullPairHamiltonian(dims, terms_from(golden, "small", rb.LocalTerm),
                                       left_axes=tuple(golden["small_left"]), right_axes=tuple(golden["small_right"]))
    bp = BatchedPropagator([h], krylov_dimension=16)
    with pytest.raises(ValueError):
        bp.propagate(golden["small_psi0"], [0.2, 0.1])


def test_shape_groups_in_caller_order(rb):
    """propagate_device on an interleaved order (one launch group per run of one shape) gives the
    same populations as propagate, which orders trajectories by shape first."""
    import torch

    from rpm_b200 import synthetic
    from rpm_b200.batched import BatchedPropagator

    full = synthetic.full_system()
    systems = [synthetic.prefix_system(full, 3), synthetic.prefix_system(full, 5)]
    hams = [rb.CompiledFullPairHamiltonian(s.dimensions, s.terms(0.5, 0.1), left_axes=s.left_axes,
                                           right_axes=s.right_axes) for s in systems]
    assert [h._system.fast_hpsi for h in hams] == [False, True]
    idx = np.array([1, 0, 1, 0], dtype=np.int32)
    psi = [synthetic.random_phase_vectors(systems[k].dimensions, 1, 300 + b)[0] for b, k in enumerate(idx)]
    times = np.arange(81) * 0.00125
    bp = BatchedPropagator(hams, krylov_dimension=24, state_error_budget=1e-9)
    sorted_run = bp.propagate(psi, times, system_index=idx)
    buf = bp.load_states(psi, idx)
    values, _, _ = bp.propagate_device(buf, times, idx)
    np.testing.assert_allclose(values.cpu().numpy(), sorted_run.observable_values, atol=2e-6)
    assert torch.isfinite(buf).all()
