"""Pin the CPU oracle against outputs of the reference implementation itself.

The fixtures in tests/golden/reference_golden.npz were produced by running the
reference (tests/golden/make_golden.py).  These tests need no GPU.
"""

import math

import numpy as np
import pytest

import oracle
from conftest import terms_from


def test_spin_operators_and_local_operators(golden):
    for s in (0.5, 1.0, 1.5):
        for name, op in zip("xyz", oracle.spin_operators(s)):
            np.testing.assert_allclose(op, golden[f"spin_{s}_{name}"], atol=1e-15)
    t = golden["coupling_tensor"]
    np.testing.assert_allclose(oracle.two_spin_coupling_operator(0.5, 1.0, t), golden["coupling_half_one"], atol=1e-14)
    np.testing.assert_allclose(oracle.two_spin_coupling_operator(0.5, 0.5, t), golden["coupling_half_half"], atol=1e-14)
    np.testing.assert_allclose(oracle.quadrupole_operator(1.0, golden["quad_tensor"]), golden["quad_one"], atol=1e-14)
    np.testing.assert_allclose(oracle.efimova_hore_electron_coupling_operator(1.7, -2.3, golden["eh_axis"]),
                               golden["eh_op"], atol=1e-14)
    np.testing.assert_allclose(oracle.field_vector_mT(37.0, 50.0), golden["field_vec"], atol=1e-17)


def test_model_tables(golden):
    for key, tensor in oracle.QUADRUPOLE_TENSORS_MT.items():
        np.testing.assert_allclose(tensor, golden[f"qtensor_{key}"], atol=1e-15)
    for k, nuc in enumerate(oracle.ALL_NUCLEI):
        np.testing.assert_array_equal(nuc.tensor_mT, golden[f"hf_{k}"])
    assert oracle.SYSTEM_DIMENSIONS == (2, 2, 3, 3, 2, 2, 2, 2, 2, 3, 2, 2, 2, 2, 2, 2)
    assert math.prod(oracle.SYSTEM_DIMENSIONS) == 221184


def test_seeds_and_initial_state(golden):
    seeds = [oracle.production_sample_seed(20260731, s) for s in range(4)]
    assert seeds == [int(v) for v in golden["seeds"]]
    init = oracle.random_phase_initial_state(oracle.SYSTEM_DIMENSIONS, 20260731, 0)
    idx = golden["init_s0_checks_idx"]
    np.testing.assert_allclose(init[idx], golden["init_s0_checks_val"], atol=1e-15)


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 8, 9, 4001])
def test_simpson_matches_reference_quadrature(golden, n):
    value = oracle.simpson(golden[f"simpson_y_{n}"], golden[f"simpson_x_{n}"])
    assert value == pytest.approx(float(golden[f"simpson_v_{n}"]), rel=1e-13, abs=1e-15)


def test_yield_integral(golden):
    v = oracle.integrate_yield(golden["yield_t"], golden["yield_p"], 1.0)
    assert v == pytest.approx(float(golden["yield_v"]), rel=1e-14)


def test_simpson_cubic_exactness():
    # the reference's known answer: exp(t) t^3 weighted by exp(-t) integrates to 1/4
    t = np.linspace(0.0, 1.0, 5)
    assert oracle.integrate_yield(t, np.exp(t) * t ** 3, 1.0) == pytest.approx(0.25, abs=1e-14)


def _small_h(golden, cls=None):
    dims = tuple(int(v) for v in golden["small_dims"])
    terms = terms_from(golden, "small", oracle.LocalTerm)
    if cls == "generic":
        return oracle.MatrixFreeHamiltonian(dims, terms)
    return oracle.CompiledFullPairHamiltonian(dims, terms, left_axes=tuple(golden["small_left"]),
                                              right_axes=tuple(golden["small_right"]))


def test_small_hamiltonian_action(golden):
    hg = _small_h(golden, "generic")
    hs = _small_h(golden)
    np.testing.assert_allclose(hg.matvec(golden["small_vec"]), golden["small_hvec"], atol=1e-12)
    np.testing.assert_allclose(hs.matvec(golden["small_vec"]), golden["small_hvec_split"], atol=1e-12)
    np.testing.assert_allclose(hg.explicit_matrix(), golden["small_dense"], atol=1e-12)


@pytest.mark.parametrize("tag,knobs", [
    ("default", {}),
    ("cfg0", dict(minimum_dimension=30, maximum_dimension=30, state_error_budget=1e-10)),
    ("cfg1", dict(minimum_dimension=8, maximum_dimension=40, state_error_budget=1e-10)),
])
def test_small_propagation_matches_reference(golden, tag, knobs):
    h = _small_h(golden)
    dims = tuple(int(v) for v in golden["small_dims"])
    prop = oracle.AdaptiveLanczosPropagator(h, **knobs)
    res = prop.propagate(golden["small_psi0"][0], golden["small_times"], oracle.SingletPopulationObservable(dims))
    np.testing.assert_allclose(res.observable_values, golden[f"small_{tag}_values"], atol=1e-11)
    # error estimates: relative where they are resolved, absolute floor at round-off level
    np.testing.assert_allclose(res.state_error_estimates, golden[f"small_{tag}_state_errors"], rtol=1e-6, atol=1e-13)
    np.testing.assert_allclose(res.final_state, golden[f"small_{tag}_final"], atol=1e-10)
    st = golden[f"small_{tag}_stats"]
    s = res.stats
    assert (s.accepted_steps, s.rejected_steps, s.matvecs, s.maximum_krylov_dimension) == tuple(int(v) for v in st[:4])
    y = oracle.integrate_yield(golden["small_times"], res.observable_values, 1.0)
    assert y == pytest.approx(float(golden[f"small_{tag}_yield"]), abs=1e-11)


def test_direct_observable_with_stored_states(golden):
    h = _small_h(golden)
    prop = oracle.AdaptiveLanczosPropagator(h, minimum_dimension=8, maximum_dimension=16, state_error_budget=1e-9)
    res = prop.propagate(golden["small_psi0"][1], golden["small_times"][:41], lambda v: float(abs(v[5]) ** 2),
                         store_states=True)
    np.testing.assert_allclose(res.observable_values, golden["small_direct_values"], atol=1e-12)
    np.testing.assert_allclose(res.states, golden["small_direct_states"], atol=1e-10)


@pytest.mark.parametrize("key", ["prefix6", "prefix10"])
def test_prefix_systems(golden, key):
    dims = tuple(int(v) for v in golden[f"{key}_dims"])
    terms = terms_from(golden, key, oracle.LocalTerm)
    h = oracle.CompiledFullPairHamiltonian(dims, terms, left_axes=tuple(golden[f"{key}_left"]),
                                           right_axes=tuple(golden[f"{key}_right"]))
    hv = h.matvec(golden[f"{key}_psi0"])
    assert float(np.vdot(hv, hv).real) == pytest.approx(float(golden[f"{key}_hvec_norm2"]), rel=1e-12)
    idx = golden[f"{key}_hvec_sample_idx"]
    np.testing.assert_allclose(hv[idx], golden[f"{key}_hvec_sample_val"], atol=1e-10)
    prop = oracle.AdaptiveLanczosPropagator(h, minimum_dimension=8, maximum_dimension=40, state_error_budget=1e-10)
    res = prop.propagate(golden[f"{key}_psi0"], golden[f"{key}_times"], oracle.SingletPopulationObservable(dims))
    np.testing.assert_allclose(res.observable_values, golden[f"{key}_values"], atol=1e-11)
    st = golden[f"{key}_stats"]
    assert (res.stats.accepted_steps, res.stats.rejected_steps, res.stats.matvecs,
            res.stats.maximum_krylov_dimension) == tuple(int(v) for v in st)


def test_production_full_size_action_and_short_propagation(golden):
    h = oracle.build_hamiltonian(0.0, 0.05, quadrupole_scale=1.0, exchange_J_uT=oracle.R2_D_PAPER_UT / -3.0,
                                 d_paper_uT=oracle.R2_D_PAPER_UT)
    init = oracle.random_phase_initial_state(oracle.SYSTEM_DIMENSIONS, 20260731, 0)
    hv = h.matvec(init)
    assert float(np.vdot(hv, hv).real) == pytest.approx(float(golden["prod_hvec_norm2"]), rel=1e-12)
    idx = golden["prod_hvec_sample_idx"]
    np.testing.assert_allclose(hv[idx], golden["prod_hvec_sample_val"], atol=1e-9)
    prop = oracle.AdaptiveLanczosPropagator(h)
    res = prop.propagate(init, golden["prod_times"], oracle.SingletPopulationObservable(oracle.SYSTEM_DIMENSIONS))
    np.testing.assert_allclose(res.observable_values, golden["prod_values"], atol=1e-11)
    assert (res.stats.accepted_steps, res.stats.rejected_steps, res.stats.matvecs) == tuple(
        int(v) for v in golden["prod_stats"][:3])
