"""Segment propagation (instantaneous pulses, piecewise-constant fields) vs the oracle."""

import math

import numpy as np
import pytest
import scipy.linalg

import oracle

pytestmark = pytest.mark.gpu

KNOBS = dict(minimum_dimension=8, maximum_dimension=24, dimension_increment=8)


def _pair(system, theta, phi, **kw):
    import rpm_b200 as rb

    terms = system.terms(theta, phi, **kw)
    h = rb.CompiledFullPairHamiltonian(system.dimensions, terms, left_axes=system.left_axes,
                                       right_axes=system.right_axes)
    ho = oracle.CompiledFullPairHamiltonian(system.dimensions, [oracle.LocalTerm(t.axes, t.operator) for t in terms],
                                            left_axes=system.left_axes, right_axes=system.right_axes)
    return h, ho


def test_local_unitary_apply_matches_oracle():
    from rpm_b200 import segments, synthetic

    sysm = synthetic.small_system()
    psi = synthetic.random_phase_vectors(sysm.dimensions, 1, 3)[0]
    u = segments.spin_pi_pulse(1.0, [0.3, 0.1, 0.9])
    got = segments.local_unitary_apply(psi, sysm.dimensions, 2, u)
    np.testing.assert_allclose(got, oracle.local_unitary_apply(psi, sysm.dimensions, 2, u), atol=1e-14)
    ref_u = scipy.linalg.expm(-1j * math.pi * sum(c * op for c, op in zip(
        np.array([0.3, 0.1, 0.9]) / np.linalg.norm([0.3, 0.1, 0.9]), oracle.spin_operators(1.0))))
    np.testing.assert_allclose(u, ref_u, atol=1e-13)


def test_periodic_pi_pulses_match_oracle():
    from rpm_b200 import segments, synthetic

    sysm = synthetic.small_system()
    h, ho = _pair(sysm, 0.4, 0.0)
    psi = synthetic.random_phase_vectors(sysm.dimensions, 1, 5)[0]
    times = np.arange(241) * 0.00125  # 0 .. 0.3 us
    u = segments.spin_pi_pulse(1.0, [0.0, 0.0, 1.0])
    ends = [0.05, 0.13, 0.21, 0.3]
    segs = [segments.Segment(e, h, (2, u)) for e in ends]
    got = segments.propagate_segments(psi, times, segs, state_error_budget=1e-9, **KNOBS)
    ref = oracle.propagate_segments(psi, times, [(e, ho, (2, u)) for e in ends], state_error_budget=1e-9, **KNOBS)
    np.testing.assert_allclose(got.observable_values, ref[0], atol=1e-11)
    np.testing.assert_allclose(got.observable_error_bounds, ref[1], rtol=1e-6, atol=1e-13)
    np.testing.assert_allclose(got.final_state, ref[2], atol=1e-10)
    assert (got.accepted_steps, got.rejected_steps, got.matvecs) == ref[3]


def test_square_field_pulse_matches_oracle():
    from rpm_b200 import segments, synthetic

    sysm = synthetic.small_system()
    h0, ho0 = _pair(sysm, 0.0, 0.0)
    h1, ho1 = _pair(sysm, 0.0, 0.0, extra_field_mT=[4e-4, 0.0, 0.0])  # 400 nT transverse
    psi = synthetic.random_phase_vectors(sysm.dimensions, 1, 9)[0]
    times = np.arange(321) * 0.00125  # 0 .. 0.4 us
    segs = segments.square_pulse_segments(h0, h1, 0.1, 0.15, 0.4)
    got = segments.propagate_segments(psi, times, segs, state_error_budget=1e-9, **KNOBS)
    ref = oracle.propagate_segments(psi, times, [(0.1, ho0, None), (0.25, ho1, None), (0.4, ho0, None)],
                                    state_error_budget=1e-9, **KNOBS)
    np.testing.assert_allclose(got.observable_values, ref[0], atol=1e-11)
    assert (got.accepted_steps, got.rejected_steps, got.matvecs) == ref[3]
    y_got = oracle.integrate_yield(times, got.observable_values, 1.0)
    assert abs(y_got - oracle.integrate_yield(times, ref[0], 1.0)) < 1e-11


def test_batched_square_pulse_matches_plain_segments():
    """Config-3-style transverse square pulse with a per-trajectory amplitude, batched vs plain FP64."""
    import rpm_b200 as rb
    from rpm_b200 import segments, synthetic
    from rpm_b200.batched import BatchedSegment, propagate_segments_batched

    sysm = synthetic.prefix_system(synthetic.full_system(), 5)
    theta, phi = 0.6, 0.0
    amps_nT = (0.0, 250.0, 500.0)
    transverse = np.array([math.cos(theta), 0.0, -math.sin(theta)])  # perpendicular to the static field in zx
    h0 = rb.CompiledFullPairHamiltonian(sysm.dimensions, sysm.terms(theta, phi), left_axes=sysm.left_axes,
                                        right_axes=sysm.right_axes)
    hp = [rb.CompiledFullPairHamiltonian(sysm.dimensions, sysm.terms(theta, phi, extra_field_mT=a * 1e-6 * transverse),
                                         left_axes=sysm.left_axes, right_axes=sysm.right_axes) for a in amps_nT]
    assert h0._system.fast_hpsi
    psi = synthetic.random_phase_vectors(sysm.dimensions, len(amps_nT), 21)
    times = np.arange(321) * 0.00125  # 0 .. 0.4 us; pulse on [0.1, 0.25)
    start, dur = 0.1, 0.15
    nb = len(amps_nT)
    segs = [BatchedSegment(start, [h0], [0] * nb), BatchedSegment(start + dur, hp, list(range(nb))),
            BatchedSegment(times[-1], [h0], [0] * nb)]
    out = propagate_segments_batched(list(psi), times, segs, state_error_budget=1e-8, lifetime_us=1.0,
                                     krylov_dimension=32)
    for b, a in enumerate(amps_nT):
        ref = segments.propagate_segments(psi[b], times, segments.square_pulse_segments(h0, hp[b], start, dur, times[-1]),
                                          state_error_budget=1e-10, **KNOBS)
        assert np.max(np.abs(out.observable_values[b] - ref.observable_values)) < 1e-5
        assert abs(out.yields[b] - rb.integrate_yield(times, ref.observable_values, 1.0)) < 1e-6
    # the pulse changes the dynamics: trajectories differ only through it
    assert np.max(np.abs(out.observable_values[2] - out.observable_values[0])) > 1e-4 or amps_nT[2] == 0.0


def test_batched_periodic_pi_pulses_match_plain_segments():
    import rpm_b200 as rb
    from rpm_b200 import segments, synthetic
    from rpm_b200.batched import BatchedSegment, propagate_segments_batched

    sysm = synthetic.prefix_system(synthetic.full_system(), 5)
    h = rb.CompiledFullPairHamiltonian(sysm.dimensions, sysm.terms(0.9, 0.3), left_axes=sysm.left_axes,
                                       right_axes=sysm.right_axes)
    psi = synthetic.random_phase_vectors(sysm.dimensions, 2, 8)
    times = np.arange(241) * 0.00125
    u = segments.spin_pi_pulse(1.0, [0.0, 0.2, 1.0])
    ends = [0.05, 0.13, 0.21, 0.3]
    out = propagate_segments_batched(list(psi), times, [BatchedSegment(e, [h], [0, 0], (2, u)) for e in ends],
                                     state_error_budget=1e-8, lifetime_us=1.0)
    for b in range(2):
        ref = segments.propagate_segments(psi[b], times, [segments.Segment(e, h, (2, u)) for e in ends],
                                          state_error_budget=1e-10, **KNOBS)
        assert np.max(np.abs(out.observable_values[b] - ref.observable_values)) < 1e-5
        assert abs(out.yields[b] - rb.integrate_yield(times, ref.observable_values, 1.0)) < 1e-6
