"""Host-side pieces of segment propagation (no GPU): pi pulses, square-pulse
segment lists, and the argument checks made before any device work."""

import math

import numpy as np
import pytest
from scipy.linalg import expm


@pytest.mark.parametrize("spin", [0.5, 1.0])
def test_spin_pi_pulse_is_the_rotation_by_pi(spin):
    from rpm_b200.model import spin_operators
    from rpm_b200.segments import spin_pi_pulse

    axis = np.array([0.3, -0.5, 0.8])
    u = spin_pi_pulse(spin, axis)
    n = axis / np.linalg.norm(axis)
    gen = sum(c * op for c, op in zip(n, spin_operators(spin)))
    np.testing.assert_allclose(u, expm(-1j * math.pi * gen), atol=1e-12)
    np.testing.assert_allclose(u @ u.conj().T, np.eye(u.shape[0]), atol=1e-12)
    if spin == 0.5:  # exp(-i pi n.sigma / 2) = -i n.sigma
        np.testing.assert_allclose(u, -2j * gen, atol=1e-12)


def test_square_pulse_segments_cover_the_horizon():
    from rpm_b200.segments import square_pulse_segments

    hs, hp = object(), object()
    segs = square_pulse_segments(hs, hp, 0.2, 0.5, 1.0)
    assert [(s.end_us, s.hamiltonian) for s in segs] == [(0.2, hs), (0.7, hp), (1.0, hs)]
    assert all(s.pulse is None for s in segs)
    # a pulse from t = 0 to the end is a single segment
    assert [(s.end_us, s.hamiltonian) for s in square_pulse_segments(hs, hp, 0.0, 1.0, 1.0)] == [(1.0, hp)]


class _Stub:
    dimensions = (2, 2, 2)


@pytest.mark.parametrize("times, ends, message", [
    ([0.1, 0.2], [0.2], "start at 0"),
    ([0.0, 0.2, 0.1], [0.1], "start at 0"),
    ([0.0, 0.1, 0.2], [0.1], "last segment"),
    ([0.0, 0.1, 0.2], [0.15, 0.1, 0.2], "strictly increasing"),
    ([0.0, 0.1, 0.2], [0.0, 0.2], "strictly increasing"),
])
def test_propagate_segments_checks_its_arguments_first(times, ends, message):
    from rpm_b200.segments import Segment, propagate_segments

    segs = [Segment(e, _Stub()) for e in ends]
    with pytest.raises(ValueError, match=message):
        propagate_segments(np.zeros(8, dtype=complex), times, segs)
