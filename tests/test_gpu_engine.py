"""GPU parity of the plain FP64 path against the reference (fixtures) and the oracle.

Bars: complex128 H psi within 1e-12 relative of the reference; propagation
decisions (accepted/rejected steps, matvecs, Krylov dimensions) identical to
the reference's and populations within 1e-11 absolute.
"""

import math

import numpy as np
import pytest
import scipy.linalg

import oracle
from conftest import terms_from

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rb():
    import rpm_b200

    return rpm_b200


def _dims(golden, key):
    return tuple(int(v) for v in golden[f"{key}_dims"])


def _h(rb, golden, key, generic=False):
    terms = terms_from(golden, key, rb.LocalTerm)
    if generic:
        return rb.MatrixFreeHamiltonian(_dims(golden, key), terms, _split=False)
    return rb.CompiledFullPairHamiltonian(_dims(golden, key), terms, left_axes=tuple(golden[f"{key}_left"]),
                                          right_axes=tuple(golden[f"{key}_right"]))


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


# --- Hamiltonian action -------------------------------------------------------

def test_small_action_generic_and_split(rb, golden):
    for generic in (True, False):
        h = _h(rb, golden, "small", generic)
        assert _rel(h.matvec(golden["small_vec"]), golden["small_hvec"]) < 1e-13
        np.testing.assert_allclose(h.explicit_matrix(), golden["small_dense"], atol=1e-12)
    h = rb.MatrixFreeHamiltonian(_dims(golden, "small"), terms_from(golden, "small", rb.LocalTerm))
    assert h._system.split  # auto-detected radical split
    assert _rel(h.matvec(golden["small_vec"]), golden["small_hvec"]) < 1e-13
    assert h.matvec_count == 1


def test_local_terms_match_dense_kronecker_products(rb):
    sx = rb.spin_operators(0.5)[0]
    sy1 = rb.spin_operators(1.0)[1]
    sz = rb.spin_operators(0.5)[2]
    terms = (rb.LocalTerm((0, 2), np.kron(sx, sz), "nonadjacent coupling"), rb.LocalTerm((1,), sy1, "middle spin"))
    h = rb.MatrixFreeHamiltonian((2, 3, 2), terms)
    expected = np.kron(sx, np.kron(np.eye(3), sz)) + np.kron(np.eye(2), np.kron(sy1, np.eye(2)))
    np.testing.assert_allclose(h.explicit_matrix(), expected, atol=1e-13)
    v = np.random.default_rng(1).normal(size=12) + 1j * np.random.default_rng(2).normal(size=12)
    assert _rel(h.matvec(v), expected @ v) < 1e-12


@pytest.mark.parametrize("key", ["prefix6", "prefix10"])
def test_prefix_action(rb, golden, key):
    h = _h(rb, golden, key)
    hv = h.matvec(golden[f"{key}_psi0"])
    assert float(np.vdot(hv, hv).real) == pytest.approx(float(golden[f"{key}_hvec_norm2"]), rel=1e-12)
    np.testing.assert_allclose(hv[golden[f"{key}_hvec_sample_idx"]], golden[f"{key}_hvec_sample_val"], atol=1e-10)
    generic = _h(rb, golden, key, generic=True)
    assert _rel(generic.matvec(golden[f"{key}_psi0"]), hv) < 1e-13


def test_full_size_synthetic_action(rb, golden):
    from rpm_b200 import synthetic

    full = synthetic.full_system()
    terms = full.terms(math.pi / 4, 0.0)
    h = rb.CompiledFullPairHamiltonian(full.dimensions, terms, left_axes=full.left_axes, right_axes=full.right_axes)
    v = synthetic.random_phase_vectors(full.dimensions, 1, 2024)[0]
    hv = h.matvec(v)
    assert float(np.vdot(hv, hv).real) == pytest.approx(float(golden["full_hvec_norm2"]), rel=1e-12)
    idx = golden["full_hvec_sample_idx"]
    np.testing.assert_allclose(hv[idx], golden["full_hvec_sample_val"], rtol=0, atol=1e-10 * np.abs(hv).max())
    probe = np.random.default_rng(7)
    pv = probe.normal(size=v.size) + 1j * probe.normal(size=v.size)
    assert abs(np.vdot(pv, hv) - golden["full_hvec_probe_dot"]) < 1e-11 * abs(golden["full_hvec_probe_dot"]) + 1e-9
    # the generic per-term kernel gives the same operator
    hg = rb.MatrixFreeHamiltonian(full.dimensions, terms, _split=False)
    assert _rel(hg.matvec(v), hv) < 1e-13
    # complex64 kernels: FP32 storage and accumulation, ~1e-7 relative
    import torch

    x = torch.from_numpy(v).to("cuda", torch.complex64)
    y = torch.empty_like(x)
    h.apply(x, y, precision=64)
    assert _rel(y.cpu().numpy(), hv) < 2e-6


def test_production_full_size_action(rb, golden):
    h = rb.build_hamiltonian(0.0, 0.05)
    init = rb.random_phase_initial_state(h.dimensions, 20260731, 0)
    hv = h.matvec(init)
    assert float(np.vdot(hv, hv).real) == pytest.approx(float(golden["prod_hvec_norm2"]), rel=1e-12)
    np.testing.assert_allclose(hv[golden["prod_hvec_sample_idx"]], golden["prod_hvec_sample_val"], atol=1e-9)


def test_batched_matmat(rb, golden):
    h = _h(rb, golden, "prefix10")
    rng = np.random.default_rng(3)
    m = rng.normal(size=(h.dimension, 5)) + 1j * rng.normal(size=(h.dimension, 5))
    out = h.matmat(m)
    for j in range(5):
        assert _rel(out[:, j], h.matvec(m[:, j])) < 1e-14


# --- Lanczos propagation ------------------------------------------------------

def _lanczos_fixture(rb):
    sx, sy, sz = rb.spin_operators(0.5)
    terms = (rb.LocalTerm((0,), 0.7 * sx + 0.2 * sz), rb.LocalTerm((1, 2), 0.4 * np.kron(sy, sx) + 0.3 * np.kron(sz, sz)))
    h = rb.MatrixFreeHamiltonian((2, 2, 2), terms)
    state = rb.singlet_initial_state((2, 2, 2), np.random.default_rng(6))
    return h, state, h.explicit_matrix()


def test_lanczos_matches_dense_exponential(rb):
    h, state, dense = _lanczos_fixture(rb)
    times = np.array([0.0, 0.03, 0.2, 0.7])
    prop = rb.AdaptiveLanczosPropagator(h, minimum_dimension=5, maximum_dimension=8, dimension_increment=1,
                                        embedded_offset=2, state_error_budget=1e-11, initial_step_us=0.4,
                                        maximum_step_us=0.4)
    res = prop.propagate(state, times, lambda v: oracle.singlet_population(v, (2, 2, 2)), store_states=True)
    expected = [oracle.singlet_population(scipy.linalg.expm(-1j * dense * t) @ state, (2, 2, 2)) for t in times]
    np.testing.assert_allclose(res.observable_values, expected, atol=2e-12)
    np.testing.assert_allclose(res.final_state, scipy.linalg.expm(-1j * dense * times[-1]) @ state, atol=2e-12)
    np.testing.assert_allclose(res.states[-1], res.final_state, atol=2e-12)
    assert res.stats.maximum_norm_error < 2e-12


def test_minimum_step_failure_is_reported(rb):
    h, state, _ = _lanczos_fixture(rb)
    prop = rb.AdaptiveLanczosPropagator(h, minimum_dimension=3, maximum_dimension=3, dimension_increment=1,
                                        embedded_offset=1, state_error_budget=1e-30, initial_step_us=1.0,
                                        maximum_step_us=1.0, minimum_step_us=0.2)
    with pytest.raises(RuntimeError):
        prop.propagate(state, [1.0], lambda v: oracle.singlet_population(v, (2, 2, 2)))


def test_rejected_step_can_recover(rb):
    h, state, _ = _lanczos_fixture(rb)
    prop = rb.AdaptiveLanczosPropagator(h, minimum_dimension=3, maximum_dimension=3, dimension_increment=1,
                                        embedded_offset=1, state_error_budget=1e-2, initial_step_us=1.0,
                                        maximum_step_us=1.0, minimum_step_us=1e-6)
    res = prop.propagate(state, [1.0], lambda v: oracle.singlet_population(v, (2, 2, 2)))
    assert res.stats.rejected_steps > 0 and res.stats.accepted_steps > 0


def test_maximum_basis_is_reused_after_growth(rb):
    rng = np.random.default_rng(4)
    values = rng.normal(size=(16, 16)) + 1j * rng.normal(size=(16, 16))
    dense = 20.0 * (values + values.conj().T) / 2.0
    h = rb.MatrixFreeHamiltonian((2, 2, 2, 2), (rb.LocalTerm((0, 1, 2, 3), dense),))
    state = rng.normal(size=16) + 1j * rng.normal(size=16)
    state /= np.linalg.norm(state)
    res = rb.AdaptiveLanczosPropagator(h, minimum_dimension=4, maximum_dimension=12, dimension_increment=4,
                                       embedded_offset=2, state_error_budget=1e-4, initial_step_us=0.1,
                                       maximum_step_us=0.1, minimum_step_us=1e-8).propagate(
        state, [0.2], lambda v: float(abs(v[0]) ** 2))
    attempts = res.stats.accepted_steps + res.stats.rejected_steps
    assert res.stats.maximum_krylov_dimension == 12
    assert res.stats.matvecs < attempts * (4 + 12)


def test_zero_vector_and_bad_times_raise(rb):
    h, state, _ = _lanczos_fixture(rb)
    prop = rb.AdaptiveLanczosPropagator(h, minimum_dimension=3, maximum_dimension=4, embedded_offset=1)
    with pytest.raises(ValueError):
        prop.propagate(np.zeros(8), [0.1], lambda v: 0.0)
    with pytest.raises(ValueError):
        prop.propagate(state, [0.2, 0.1], lambda v: 0.0)
    with pytest.raises(ValueError):
        prop.propagate(state[:4], [0.1], lambda v: 0.0)


@pytest.mark.parametrize("tag,knobs", [
    ("default", {}),
    ("cfg0", dict(minimum_dimension=30, maximum_dimension=30, state_error_budget=1e-10)),
    ("cfg1", dict(minimum_dimension=8, maximum_dimension=40, state_error_budget=1e-10)),
])
def test_small_propagation_matches_reference(rb, golden, tag, knobs):
    h = _h(rb, golden, "small")
    dims = _dims(golden, "small")
    res = rb.AdaptiveLanczosPropagator(h, **knobs).propagate(golden["small_psi0"][0], golden["small_times"],
                                                             rb.SingletPopulationObservable(dims))
    st = golden[f"small_{tag}_stats"]
    s = res.stats
    assert (s.accepted_steps, s.rejected_steps, s.matvecs, s.maximum_krylov_dimension) == tuple(int(v) for v in st[:4])
    np.testing.assert_allclose(res.observable_values, golden[f"small_{tag}_values"], atol=1e-11)
    np.testing.assert_allclose(res.state_error_estimates, golden[f"small_{tag}_state_errors"], rtol=1e-6, atol=1e-13)
    np.testing.assert_allclose(res.final_state, golden[f"small_{tag}_final"], atol=1e-10)
    y = rb.integrate_yield(golden["small_times"], res.observable_values, 1.0)
    assert y == pytest.approx(float(golden[f"small_{tag}_yield"]), abs=1e-11)


def test_direct_observable_with_stored_states(rb, golden):
    h = _h(rb, golden, "small")
    prop = rb.AdaptiveLanczosPropagator(h, minimum_dimension=8, maximum_dimension=16, state_error_budget=1e-9)
    res = prop.propagate(golden["small_psi0"][1], golden["small_times"][:41], lambda v: float(abs(v[5]) ** 2),
                         store_states=True)
    np.testing.assert_allclose(res.observable_values, golden["small_direct_values"], atol=1e-12)
    np.testing.assert_allclose(res.states, golden["small_direct_states"], atol=1e-10)
    assert (res.stats.accepted_steps, res.stats.rejected_steps, res.stats.matvecs) == tuple(
        int(v) for v in golden["small_direct_stats"])


@pytest.mark.parametrize("key", ["prefix6", "prefix10"])
def test_prefix_propagation_matches_reference(rb, golden, key):
    h = _h(rb, golden, key)
    res = rb.AdaptiveLanczosPropagator(h, minimum_dimension=8, maximum_dimension=40, state_error_budget=1e-10).propagate(
        golden[f"{key}_psi0"], golden[f"{key}_times"], rb.SingletPopulationObservable(_dims(golden, key)))
    np.testing.assert_allclose(res.observable_values, golden[f"{key}_values"], atol=1e-11)
    assert (res.stats.accepted_steps, res.stats.rejected_steps, res.stats.matvecs,
            res.stats.maximum_krylov_dimension) == tuple(int(v) for v in golden[f"{key}_stats"])
    assert float(np.vdot(res.final_state, res.final_state).real) == pytest.approx(
        float(golden[f"{key}_final_norm2"]), abs=1e-12)
    idx = golden[f"{key}_final_sample_idx"]
    np.testing.assert_allclose(res.final_state[idx], golden[f"{key}_final_sample_val"], atol=1e-10)


def test_production_short_propagation_matches_reference(rb, golden):
    h = rb.build_hamiltonian(0.0, 0.05)
    init = rb.random_phase_initial_state(h.dimensions, 20260731, 0)
    res = rb.make_propagator(h).propagate(init, golden["prod_times"], rb.SingletPopulationObservable(h.dimensions))
    np.testing.assert_allclose(res.observable_values, golden["prod_values"], atol=1e-11)
    assert (res.stats.accepted_steps, res.stats.rejected_steps, res.stats.matvecs) == tuple(
        int(v) for v in golden["prod_stats"][:3])
    idx = golden["prod_final_sample_idx"]
    np.testing.assert_allclose(res.final_state[idx], golden["prod_final_sample_val"], atol=1e-10)


def test_matches_oracle_on_medium_horizon(rb, golden):
    # oracle (CPU) vs GPU on the 864-dim system over 0.25 us at the config-1 knobs
    key = "prefix6"
    dims = _dims(golden, key)
    t_ref = terms_from(golden, key, oracle.LocalTerm)
    href = oracle.CompiledFullPairHamiltonian(dims, t_ref, left_axes=tuple(golden[f"{key}_left"]),
                                              right_axes=tuple(golden[f"{key}_right"]))
    times = np.arange(201) * 0.00125
    knobs = dict(minimum_dimension=8, maximum_dimension=40, state_error_budget=1e-10)
    ref = oracle.AdaptiveLanczosPropagator(href, **knobs).propagate(golden[f"{key}_psi0"], times,
                                                                   oracle.SingletPopulationObservable(dims))
    got = rb.AdaptiveLanczosPropagator(_h(rb, golden, key), **knobs).propagate(
        golden[f"{key}_psi0"], times, rb.SingletPopulationObservable(dims))
    np.testing.assert_allclose(got.observable_values, ref.observable_values, atol=1e-11)
    assert got.stats.matvecs == ref.stats.matvecs
    yr = oracle.integrate_yield(times, ref.observable_values, 1.0)
    yg = rb.integrate_yield(times, got.observable_values, 1.0)
    assert abs(yr - yg) < 1e-11


# --- yield and observables ----------------------------------------------------

@pytest.mark.parametrize("n", [2, 3, 4, 5, 8, 9, 4001])
def test_gpu_simpson_matches_reference(rb, golden, n):
    x, y = golden[f"simpson_x_{n}"], golden[f"simpson_y_{n}"]
    # integrate_yield(t, P, tau) integrates exp(-t/tau) P / tau; undo the weight with tau -> large
    tau = 1e300
    got = rb.integrate_yield(x, y * tau, tau)
    assert got == pytest.approx(float(golden[f"simpson_v_{n}"]), rel=1e-12, abs=1e-14)


def test_gpu_yield_integral(rb, golden):
    assert rb.integrate_yield(golden["yield_t"], golden["yield_p"], 1.0) == pytest.approx(float(golden["yield_v"]),
                                                                                         rel=1e-14)
    t = np.linspace(0.0, 1.0, 5)
    assert rb.integrate_yield(t, np.exp(t) * t ** 3, 1.0) == pytest.approx(0.25, abs=1e-14)


def test_singlet_population_matches_dense_projector(rb):
    dims = (2, 2, 3)
    rng = np.random.default_rng(4)
    state = rng.normal(size=12) + 1j * rng.normal(size=12)
    state /= np.linalg.norm(state)
    singlet = np.array([0.0, 1.0, -1.0, 0.0]) / np.sqrt(2.0)
    projector = np.kron(np.outer(singlet, singlet), np.eye(3))
    assert rb.singlet_population(state, dims) == pytest.approx(float(np.vdot(state, projector @ state).real), abs=1e-14)
    obs = rb.SingletPopulationObservable(dims)
    basis = rng.normal(size=(12, 4)) + 1j * rng.normal(size=(12, 4))
    ref = oracle.SingletPopulationObservable(dims).project_basis(basis)
    np.testing.assert_allclose(obs.project_basis(basis), ref, atol=1e-13)
