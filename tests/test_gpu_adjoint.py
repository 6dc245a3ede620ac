"""Adjoint gradients of the singlet yield vs central differences of FP64 yields.

Parameters (rpm_b200.adjoint.PARAMETERS): static field |B| (uT), its polar and
azimuthal angles (rad), the amplitude of a transverse square pulse (nT) and a
global hyperfine scale.  Central differences use the relative step 1e-4 of
the benchmark specification (with Richardson extrapolation where the
yields are exact to rounding), through exact dense propagation (864 and 96
dimensions) or, at 221,184 dimensions, the fixed-schedule FP64 forward of
the adjoint engine and the plain FP64 Krylov segment path.  Every gradient
component must be within GRAD_RTOL of its difference quotient.
"""

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

PARAMS = np.array([50.0, 0.7, 0.3, 300.0, 1.0])
GRAD_RTOL = 1e-4
FIELD = slice(0, 4)  # |B|, theta, phi, pulse amplitude


def _dense(system, terms):
    h = oracle.MatrixFreeHamiltonian(system.dimensions, [oracle.LocalTerm(t.axes, t.operator) for t in terms])
    return h.explicit_matrix()


def _dense_yield(system, model, psi, times, p, lifetime=1.0):
    b, th, ph, _, sc = p
    hs = _dense(system, system.terms(th, ph, field_microT=b, hyperfine_scale=sc))
    hp = _dense(system, system.terms(th, ph, field_microT=b, hyperfine_scale=sc, extra_field_mT=model.pulse_field_mT(p)))
    start = model.pulse_start_us
    return oracle.pulsed_yield_dense(hs, hp, system.dimensions, psi, times, start, start + model.pulse_duration_us,
                                     lifetime)[1]


def _check(got, ref, rtol=GRAD_RTOL):
    err = np.abs(got - ref)
    assert np.all(err <= rtol * np.abs(ref)), (got, ref, err / np.abs(ref))


def _case(prefix):
    from rpm_b200 import adjoint, synthetic

    system = synthetic.small_system() if prefix is None else synthetic.prefix_system(synthetic.full_system(), prefix)
    model = adjoint.ParametricRadicalPair(system, pulse_start_us=0.05, pulse_duration_us=0.1)
    times = np.arange(201) * 0.00125  # 0 .. 0.25 us
    psi = synthetic.random_phase_vectors(system.dimensions, 2, 11)
    return system, model, times, psi


@pytest.mark.parametrize("prefix", [None, 3])
def test_complex128_gradients_match_dense_central_differences(prefix):
    from rpm_b200 import adjoint

    system, model, times, psi = _case(prefix)
    res = adjoint.AdjointYieldGradient(model, precision="c128", checkpoint_intervals=64)(PARAMS, list(psi), times, 1.0)
    assert res.diagnostics["max_taylor_tail"] < 1e-9
    assert res.diagnostics["checkpoint_drift"] < 1e-9
    for b in range(len(psi)):
        f = lambda p: _dense_yield(system, model, psi[b], times, p)
        assert abs(res.yields[b] - f(PARAMS)) < 1e-9
        _check(res.gradients[b], oracle.central_difference(f, PARAMS, richardson=True))


@pytest.mark.parametrize("prefix", [None, 3])
def test_complex64_field_gradients_match_dense_central_differences(prefix):
    """The complex64 path (batched Krylov forward, complex64 Taylor basis):
    field derivatives are well conditioned; the hyperfine-scale derivative is
    only reported to the complex64 state floor (checked loosely)."""
    from rpm_b200 import adjoint

    system, model, times, psi = _case(prefix)
    res = adjoint.AdjointYieldGradient(model, precision="c64", krylov_dimension=24,
                                       state_error_budget=1e-8)(PARAMS, list(psi), times, 1.0)
    for b in range(len(psi)):
        f = lambda p: _dense_yield(system, model, psi[b], times, p)
        assert abs(res.yields[b] - f(PARAMS)) < 1e-6
        fd = oracle.central_difference(f, PARAMS, richardson=True)
        _check(res.gradients[b, FIELD], fd[FIELD])
        _check(res.gradients[b, 4:], fd[4:], rtol=1e-2)


def test_theta_gradient_matches_the_reference_style_angle_grid():
    """np.gradient over a theta grid, the reference's own derivative of yields."""
    from rpm_b200 import adjoint

    system, model, times, psi = _case(None)
    res = adjoint.AdjointYieldGradient(model, precision="c128")(PARAMS, [psi[0]], times, 1.0)
    h = 1e-3
    thetas = PARAMS[1] + h * np.arange(-2, 3)
    yields = []
    for th in thetas:
        p = PARAMS.copy()
        p[1] = th
        yields.append(_dense_yield(system, model, psi[0], times, p))
    slope = np.gradient(np.array(yields), thetas)[2]
    assert abs(res.gradients[0, 1] - slope) < 1e-4 * abs(slope)


def test_autograd_function_contracts_the_adjoint():
    import torch

    from rpm_b200 import adjoint

    system, model, times, psi = _case(None)
    engine = adjoint.AdjointYieldGradient(model, precision="c128")
    res = engine(PARAMS, list(psi), times, 1.0)
    p = torch.tensor(PARAMS, dtype=torch.float64, requires_grad=True)
    y = adjoint.singlet_yield(p, engine, list(psi), times, 1.0)
    assert y.shape == (len(psi),)
    np.testing.assert_allclose(y.detach().cpu().numpy(), res.yields, rtol=0, atol=1e-13)
    weights = torch.tensor([1.0, -2.0], dtype=torch.float64, device=y.device)
    (y * weights).sum().backward()
    expect = weights.cpu().numpy() @ res.gradients
    np.testing.assert_allclose(p.grad.numpy(), expect, rtol=1e-9, atol=0)


def test_non_uniform_grid_is_refused():
    from rpm_b200 import adjoint

    system, model, times, psi = _case(None)
    with pytest.raises(ValueError):
        adjoint.AdjointYieldGradient(model)(PARAMS, [psi[0]], np.concatenate([times, [times[-1] + 0.01]]), 1.0)


def test_full_size_gradients_match_fp64_central_differences():
    """221,184 dimensions, one random-phase vector, 50 uT, 300 nT pulse on [0.2, 0.7] us, t to 0.8 us."""
    from rpm_b200 import adjoint, segments, synthetic

    full = synthetic.full_system()
    model = adjoint.ParametricRadicalPair(full, pulse_start_us=0.2, pulse_duration_us=0.5)
    times = np.arange(641) * 0.00125
    psi = synthetic.random_phase_vectors(full.dimensions, 1, 29)
    engine = adjoint.AdjointYieldGradient(model, precision="c128")
    res = engine(PARAMS, list(psi), times, 1.0)
    assert res.diagnostics["max_taylor_tail"] < 1e-9
    w = adjoint.yield_weights(times, 1.0)

    def krylov_fp64_yield(p):
        hs, hp = model.hamiltonians(p)
        segs = segments.square_pulse_segments(hs, hp, model.pulse_start_us, model.pulse_duration_us, times[-1])
        out = segments.propagate_segments(psi[0], times, segs, state_error_budget=1e-11, minimum_dimension=24,
                                          maximum_dimension=48, dimension_increment=8)
        return float(w @ out.observable_values)

    # the forward yield is the plain FP64 Krylov yield
    assert abs(res.yields[0] - krylov_fp64_yield(PARAMS)) < 1e-9
    # all five components against differences through the fixed-schedule FP64 forward
    fd = oracle.central_difference(lambda p: float(engine.yields(p, list(psi), times, 1.0)[0]), PARAMS,
                                   richardson=True)
    _check(res.gradients[0], fd)
    # the hyperfine scale also against differences through the adaptive FP64 Krylov path
    s_fd = oracle.central_difference(lambda s: krylov_fp64_yield(np.concatenate([PARAMS[:4], s])), PARAMS[4:])
    _check(res.gradients[0, 4:], s_fd)


def test_full_size_complex64_field_gradients_match_complex128():
    """221,184 dimensions, two trajectories: the complex64 path's angle and pulse derivatives against the
    complex128 adjoint (itself within 1e-4 of FP64 central differences above).  |B| (a small derivative
    here, so its absolute complex64 error is a large fraction of it) and the hyperfine scale (complex64
    states limit it) are checked loosely."""
    from rpm_b200 import adjoint, synthetic

    full = synthetic.full_system()
    model = adjoint.ParametricRadicalPair(full, pulse_start_us=0.2, pulse_duration_us=0.5)
    times = np.arange(641) * 0.00125
    psi = list(synthetic.random_phase_vectors(full.dimensions, 2, 31))
    ref = adjoint.AdjointYieldGradient(model, precision="c128")(PARAMS, psi, times, 1.0)
    got = adjoint.AdjointYieldGradient(model, precision="c64", state_error_budget=1e-8)(PARAMS, psi, times, 1.0)
    np.testing.assert_allclose(got.yields, ref.yields, rtol=0, atol=1e-6)
    for b in range(len(psi)):
        _check(got.gradients[b, 1:4], ref.gradients[b, 1:4])
        _check(got.gradients[b, :1], ref.gradients[b, :1], rtol=1e-2)
        _check(got.gradients[b, 4:], ref.gradients[b, 4:], rtol=3e-2)


def test_benchmark_scale_gradients_64_vectors_random_pulse_amplitude():
    """The differentiation workload at scale: 221,184 dimensions, 64 random-phase
    vectors, 50 uT, a transverse pulse on [0.2, 0.7] us of amplitude drawn from
    U(0, 500) nT, t to 0.8 us.  The gradient of the mean yield from the
    complex128 adjoint against central differences (relative step 1e-4) of the
    mean FP64 yield, all five parameters within 1e-4; the complex64 adjoint's
    angle and pulse-amplitude components against the complex128 ones."""
    from rpm_b200 import adjoint, synthetic

    full = synthetic.full_system()
    model = adjoint.ParametricRadicalPair(full, pulse_start_us=0.2, pulse_duration_us=0.5)
    times = np.arange(641) * 0.00125
    amplitude = float(np.random.default_rng(2024).uniform(0.0, 500.0))
    params = np.array([50.0, 0.7, 0.3, amplitude, 1.0])
    psi = list(synthetic.random_phase_vectors(full.dimensions, 64, 31))
    engine = adjoint.AdjointYieldGradient(model, precision="c128")
    res = engine(params, psi, times, 1.0)
    grad = res.gradients.mean(axis=0)
    fd = oracle.central_difference(lambda p: float(np.mean(engine.yields(p, psi, times, 1.0))), params)
    _check(grad, fd)
    fast = adjoint.AdjointYieldGradient(model, precision="c64")(params, psi, times, 1.0)
    _check(fast.gradients.mean(axis=0)[1:4], grad[1:4])
