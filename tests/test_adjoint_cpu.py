"""Host-side pieces of the adjoint gradient: quadrature weights, field derivatives, segments."""

import math

import numpy as np
import pytest

import oracle


def test_simpson_weights_reproduce_the_oracle_rule():
    from rpm_b200.adjoint import simpson_weights

    rng = np.random.default_rng(3)
    for n in (2, 3, 4, 5, 10, 11, 401):
        uniform = np.arange(n) * 0.00125
        ragged = np.concatenate([[0.0], np.cumsum(rng.uniform(0.5, 1.5, n - 1))])
        for t in (uniform, ragged):
            y = rng.standard_normal(n)
            assert abs(simpson_weights(t) @ y - oracle.simpson(y, t)) < 1e-12 * max(1.0, np.abs(y).sum())


def test_yield_weights_give_the_reference_yield():
    from rpm_b200.adjoint import yield_weights

    t = oracle.time_grid_us(0.5)
    pops = 0.25 + 0.1 * np.sin(37.0 * t)
    assert abs(yield_weights(t, 1.0) @ pops - oracle.integrate_yield(t, pops, 1.0)) < 1e-14


def test_field_derivatives_match_numerical_derivatives():
    from rpm_b200 import synthetic
    from rpm_b200.adjoint import ParametricRadicalPair

    model = ParametricRadicalPair(synthetic.small_system())
    p = np.array([50.0, 0.7, 0.3, 300.0, 1.0])
    d = model.field_derivatives_mT(p)
    for seg in (0, 1):
        for i in range(5):
            h = 1e-6 * max(abs(p[i]), 1.0)
            up, down = p.copy(), p.copy()
            up[i] += h
            down[i] -= h
            num = (model.field_mT(up)[seg] - model.field_mT(down)[seg]) / (2 * h)
            np.testing.assert_allclose(d[seg, i], num, atol=1e-9 * max(1.0, np.abs(num).max()))


def test_field_of_the_pulse_is_transverse():
    from rpm_b200 import synthetic
    from rpm_b200.adjoint import ParametricRadicalPair

    model = ParametricRadicalPair(synthetic.small_system())
    p = np.array([50.0, 0.7, 0.3, 300.0, 1.0])
    static, pulsed = model.field_mT(p)
    assert abs(np.linalg.norm(static) - 0.05) < 1e-15
    assert abs(np.dot(static, pulsed - static)) < 1e-18
    assert abs(np.linalg.norm(pulsed - static) - 300e-6) < 1e-15


def test_electron_pair_zeeman_is_the_two_electron_sum():
    from rpm_b200.adjoint import electron_pair_zeeman

    b = np.array([0.01, -0.02, 0.05])
    z = oracle.TWOPI * oracle.GAMMA_E_MHZ_PER_MT * sum(c * op for c, op in zip(b, oracle.spin_operators(0.5)))
    e = electron_pair_zeeman(b)
    np.testing.assert_allclose(e, np.kron(z, np.eye(2)) + np.kron(np.eye(2), z), atol=1e-14)
    np.testing.assert_allclose(e, e.conj().T, atol=1e-14)


def test_interval_segments_follow_the_pulse_window():
    from rpm_b200 import synthetic
    from rpm_b200.adjoint import ParametricRadicalPair

    model = ParametricRadicalPair(synthetic.small_system(), pulse_start_us=0.2, pulse_duration_us=0.5)
    t = np.arange(801) * 0.00125
    seg = model.interval_segments(t)
    assert seg.size == 800
    assert seg.sum() == 400 and seg[159] == 0 and seg[160] == 1 and seg[559] == 1 and seg[560] == 0
    off_grid = ParametricRadicalPair(synthetic.small_system(), pulse_start_us=0.2001, pulse_duration_us=0.5)
    with pytest.raises(ValueError):
        off_grid.interval_segments(t)


def test_taylor_degree_meets_the_remainder_bound():
    from rpm_b200.adjoint import taylor_degree

    for x in (0.05, 0.5, 0.74, 1.5):
        d = taylor_degree(x, 1e-10)
        assert x ** (d + 1) / math.factorial(d + 1) <= 1e-10
        assert d == 1 or x ** d / math.factorial(d) > 1e-10
    with pytest.raises(ValueError):
        taylor_degree(40.0)


def test_dense_oracle_differences_pin_an_exact_derivative():
    """The oracle's central differences agree with the exact derivative of a
    discrete yield, computed through the block-triangular exponential of each
    interval (the Frechet derivative of exp)."""
    from scipy.linalg import expm

    rng = np.random.default_rng(5)
    n, dt = 8, 0.01
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    h0 = 3.0 * (a + a.conj().T)
    b = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    d = b + b.conj().T
    psi = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    psi /= np.linalg.norm(psi)
    proj = np.zeros((n, n))
    proj[1, 1] = proj[2, 2] = 0.5
    proj[1, 2] = proj[2, 1] = -0.5
    t = np.arange(41) * dt

    def phi(x):
        u = expm(-1j * (h0 + x[0] * d) * dt)
        v, pops = psi.copy(), []
        for _ in range(t.size):
            pops.append(np.vdot(v, proj @ v).real)
            v = u @ v
        return oracle.simpson(np.array(pops), t)

    big = np.zeros((2 * n, 2 * n), dtype=complex)
    big[:n, :n] = big[n:, n:] = -1j * h0 * dt
    big[:n, n:] = -1j * d * dt
    e = expm(big)
    u, du = e[:n, :n], e[:n, n:]
    v, dv, pops_d = psi.copy(), np.zeros(n, dtype=complex), []
    for _ in range(t.size):
        pops_d.append(2.0 * np.vdot(v, proj @ dv).real)
        v, dv = u @ v, u @ dv + du @ v
    exact = oracle.simpson(np.array(pops_d), t)
    assert abs(oracle.central_difference(phi, np.array([0.0]))[0] - exact) < 1e-7 * max(1.0, abs(exact))
    assert abs(oracle.central_difference(phi, np.array([0.0]), richardson=True)[0] - exact) < 1e-10 * max(1.0, abs(exact))


def test_pulsed_dense_oracle_agrees_with_the_haberkorn_oracle_without_a_pulse():
    from rpm_b200 import synthetic

    sysm = synthetic.small_system()
    terms = sysm.terms(0.4, 0.9)
    h = oracle.MatrixFreeHamiltonian(sysm.dimensions, [oracle.LocalTerm(t.axes, t.operator) for t in terms]).explicit_matrix()
    psi = synthetic.random_phase_vectors(sysm.dimensions, 1, 6)[0]
    times = np.arange(161) * 0.00125
    pops, y = oracle.pulsed_yield_dense(h, h, sysm.dimensions, psi, times, 0.05, 0.15, 0.5)
    factored, y_h = oracle.haberkorn_dense(h, sysm.dimensions, psi, times, 2.0, 2.0)
    np.testing.assert_allclose(pops, factored, atol=1e-11)
    assert abs(y - y_h) < 1e-12
