"""Persistent Lanczos kernel (one launch per Krylov step) against the
per-iteration pass launches and the FP64 plain path (GPU).

Both batched forms run the same tile arithmetic; they differ only in the
order of the FP64 partial sums of alpha/beta (per tile instead of per block),
so their populations agree far below the complex64 floor.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SAME_TOL = 1e-8   # persistent vs per-iteration passes (populations)
YIELD_TOL = 1e-6  # against the FP64 plain path


def _systems(which, norient):
    import rpm_b200 as rb
    from rpm_b200 import synthetic

    full = synthetic.full_system()
    sub = synthetic.prefix_system(full, 5) if which == "prefix" else full
    hams = [rb.CompiledFullPairHamiltonian(sub.dimensions, sub.terms(th, ph), left_axes=sub.left_axes,
                                           right_axes=sub.right_axes)
            for th, ph in synthetic.fibonacci_sphere(norient)]
    return sub, hams


def _plain_yield(rb, h, psi, times, dims):
    ref = rb.AdaptiveLanczosPropagator(h, minimum_dimension=8, maximum_dimension=40,
                                       state_error_budget=1e-10).propagate(psi, times,
                                                                           rb.SingletPopulationObservable(dims))
    return ref.observable_values, rb.integrate_yield(times, ref.observable_values, 1.0)


@pytest.mark.parametrize("warps", [8, 10])
@pytest.mark.parametrize("which,nvec,wavefront,krylov", [("prefix", 7, 3, 16), ("full", 6, 12, 16),
                                                         ("full", 5, 2, 24)])
def test_persistent_matches_pass_launches(which, nvec, wavefront, krylov, warps):
    from rpm_b200 import _lib, synthetic
    from rpm_b200.batched import BatchedPropagator

    _lib.call("rpm_set_persistent_warps", warps)

    sub, hams = _systems(which, 2)
    states = synthetic.random_phase_vectors(sub.dimensions, nvec, 11)
    index = np.arange(nvec) % len(hams)
    times = np.arange(81) * 0.00125
    out = {}
    for kind in ("persistent", "passes"):
        bp = BatchedPropagator(hams, krylov_dimension=krylov, state_error_budget=1e-8, lanczos_kernel=kind,
                               wavefront=wavefront)
        out[kind] = bp.propagate(list(states), times, system_index=index, lifetime_us=1.0)
        assert bp.lanczos_kind() == kind
        assert not np.any(out[kind].status)
    _lib.call("rpm_set_persistent_warps", 8)
    a, b = out["persistent"], out["passes"]
    assert np.max(np.abs(a.observable_values - b.observable_values)) < SAME_TOL
    assert np.max(np.abs(a.yields - b.yields)) < SAME_TOL
    for sa, sb in zip(a.stats, b.stats):
        assert abs(sa.accepted_steps - sb.accepted_steps) <= 1


def test_persistent_batch_against_fp64_plain_path():
    """Full system, three orientations whose trajectories finish at different
    Krylov steps (later launches skip finished vectors), wavefront groups of 4
    with a remainder."""
    import rpm_b200 as rb
    from rpm_b200 import synthetic
    from rpm_b200.batched import BatchedPropagator

    sub, hams = _systems("full", 3)
    nvec = 6
    states = synthetic.random_phase_vectors(sub.dimensions, nvec, 23)
    index = np.arange(nvec) % len(hams)
    times = np.arange(161) * 0.00125
    bp = BatchedPropagator(hams, krylov_dimension=32, state_error_budget=5e-8, wavefront=4,
                           lanczos_kernel="persistent")
    out = bp.propagate(list(states), times, system_index=index, lifetime_us=1.0)
    assert bp.lanczos_kind() == "persistent"
    for k in range(nvec):
        ref, y_ref = _plain_yield(rb, hams[index[k]], states[k], times, sub.dimensions)
        assert abs(out.yields[k] - y_ref) < YIELD_TOL
        assert np.max(np.abs(out.observable_values[k] - ref)) < 1e-5


@pytest.mark.parametrize("period", [4, 7])
def test_periodic_reorthogonalisation(period):
    """Periodic reorthogonalisation: persistent segments and per-iteration
    passes agree, and the yields stay on the FP64 plain path."""
    import rpm_b200 as rb
    from rpm_b200 import synthetic
    from rpm_b200.batched import BatchedPropagator

    sub, hams = _systems("prefix", 2)
    nvec = 4
    states = synthetic.random_phase_vectors(sub.dimensions, nvec, 5)
    index = np.arange(nvec) % len(hams)
    times = np.arange(161) * 0.00125
    out = {}
    for kind in ("persistent", "passes"):
        bp = BatchedPropagator(hams, krylov_dimension=24, state_error_budget=1e-8, lanczos_kernel=kind,
                               wavefront=3, reorth_period=period)
        out[kind] = bp.propagate(list(states), times, system_index=index, lifetime_us=1.0)
        assert bp.lanczos_kind() == kind
    assert np.max(np.abs(out["persistent"].observable_values - out["passes"].observable_values)) < SAME_TOL
    for k in range(nvec):
        _, y_ref = _plain_yield(rb, hams[index[k]], states[k], times, sub.dimensions)
        assert abs(out["persistent"].yields[k] - y_ref) < YIELD_TOL


def test_concurrent_batches_match_one_batch():
    """Two concurrent batches on their own streams (persistent launches that
    leave SMs free) give the single batch's results trajectory by trajectory."""
    import torch

    from rpm_b200 import synthetic
    from rpm_b200.batched import BatchedPropagator, ConcurrentBatches

    sub, hams = _systems("prefix", 3)
    nvec = 9
    states = synthetic.random_phase_vectors(sub.dimensions, nvec, 41)
    index = np.arange(nvec) % len(hams)
    times = np.arange(81) * 0.00125
    one = BatchedPropagator(hams, krylov_dimension=16, state_error_budget=1e-8)
    two = ConcurrentBatches(hams, parts=2, reserve_sms=16, krylov_dimension=16, state_error_budget=1e-8)
    ref = one.propagate(list(states), times, system_index=index, lifetime_us=1.0)
    got = two.propagate(list(states), times, system_index=index, lifetime_us=1.0)
    assert np.max(np.abs(got.observable_values - ref.observable_values)) < SAME_TOL
    assert np.max(np.abs(got.yields - ref.yields)) < SAME_TOL
    # the device-buffer path of the benchmark
    psi = one.load_states(list(states), index)
    v1, _, _ = one.propagate_device(psi.clone(), times, index)
    v2, _, _ = two.propagate_device(psi.clone(), times, index)
    torch.cuda.synchronize()
    assert float(torch.max(torch.abs(v1 - v2))) < SAME_TOL
