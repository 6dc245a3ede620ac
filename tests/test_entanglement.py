"""Entanglement observables of stored states against the reference (core.py:107-365).

Fixtures: tests/golden/entanglement_golden.npz, produced by running the
reference (tests/golden/make_entanglement_golden.py).  Bars: log negativities
within 1e-10, density matrices within 1e-12 (FP64 throughout); the cell's
propagated populations within 1e-11 (the plain path repeats the reference's
decisions).
"""

import math

import numpy as np
import pytest

import oracle

GOLDEN = np.load(__file__.rsplit("/", 1)[0] + "/golden/entanglement_golden.npz")
SPLITS = {"radical": (0, 2, 3), "electrons": (0, 1), "axis3": (3,), "mixed": (1, 2, 5)}


def test_oracle_matches_reference_fixtures():
    dims = tuple(GOLDEN["dims4"])
    for name, left in SPLITS.items():
        got = [oracle.pure_log_negativity(s, dims, left) for s in GOLDEN["states4"]]
        np.testing.assert_allclose(got, GOLDEN[f"lneg_{name}"], rtol=0, atol=1e-12)
    rho = np.array([oracle.reduced_electron_density(s, dims) for s in GOLDEN["states4"]])
    np.testing.assert_allclose(rho, GOLDEN["rho_electrons"], rtol=1e-13, atol=1e-12)
    rho_n = rho / np.trace(rho, axis1=1, axis2=2)[:, None, None]
    np.testing.assert_allclose([oracle.mixed_two_electron_log_negativity(r) for r in rho_n], GOLDEN["mixed_lneg"],
                               atol=1e-12)
    assert oracle.pure_log_negativity(GOLDEN["states4"][0], dims, (0, 1)) == pytest.approx(0.0, abs=1e-12)


def test_production_helpers_match_reference():
    from rpm_b200 import production as p

    fine, idx = p.entanglement_time_grids_us()
    np.testing.assert_array_equal(fine, GOLDEN["grid_fine"])
    np.testing.assert_array_equal(idx, GOLDEN["grid_coarse_idx"])
    for s in range(4):
        assert p.full_product_basis_indices(20260731, s) == tuple(int(v) for v in GOLDEN["product_indices"][s])
    dims = p.dimensions_for(p.selected_nuclei(4))
    assert dims == tuple(GOLDEN["dims4"])
    init = p.product_basis_initial_state(dims, p.paired_product_indices(4, p.full_product_basis_indices(20260731, 3)))
    np.testing.assert_array_equal(init, GOLDEN["states4"][0])
    with pytest.raises(ValueError):
        p.selected_nuclei(3)


def test_partial_transpose_matches_reference():
    from rpm_b200.entanglement import partial_transpose_two_qubits

    rho = GOLDEN["rho_electrons"][1]
    np.testing.assert_array_equal(partial_transpose_two_qubits(rho, 0), GOLDEN["pt0"])
    np.testing.assert_array_equal(partial_transpose_two_qubits(rho, 1), GOLDEN["pt1"])
    with pytest.raises(ValueError):
        partial_transpose_two_qubits(rho, 2)


@pytest.mark.gpu
def test_gpu_observables_match_reference():
    from rpm_b200 import entanglement as ent

    dims = tuple(GOLDEN["dims4"])
    states = GOLDEN["states4"]
    for name, left in SPLITS.items():
        np.testing.assert_allclose(ent.pure_log_negativity(states, dims, left), GOLDEN[f"lneg_{name}"], atol=1e-10)
        assert ent.pure_log_negativity(states[2], dims, left) == pytest.approx(GOLDEN[f"lneg_{name}"][2], abs=1e-10)
    rho = ent.reduced_electron_density(states, dims)
    np.testing.assert_allclose(rho, GOLDEN["rho_electrons"], rtol=1e-12, atol=1e-10)
    rho_n = rho / np.trace(rho, axis1=1, axis2=2)[:, None, None]
    np.testing.assert_allclose(ent.mixed_two_electron_log_negativity_batch(rho_n), GOLDEN["mixed_lneg"], atol=1e-10)
    assert ent.mixed_two_electron_log_negativity(rho_n[3]) == pytest.approx(GOLDEN["mixed_lneg"][3], abs=1e-10)
    # known answers of the reference's tests: product state 0, Bell state 1
    bell = np.array([1, 0, 0, 1], dtype=complex) / math.sqrt(2)
    assert ent.pure_log_negativity(bell, (2, 2), (0,)) == pytest.approx(1.0, abs=1e-12)
    assert ent.pure_log_negativity(np.array([1, 0, 0, 0], dtype=complex), (2, 2), (0,)) == pytest.approx(0.0, abs=1e-12)
    with pytest.raises(ValueError):
        ent.pure_log_negativity(np.zeros(4, dtype=complex), (2, 2), (0,))
    with pytest.raises(ValueError):
        ent.pure_log_negativity(bell, (2, 2), (0, 0))


@pytest.mark.gpu
def test_gpu_radical_split_at_full_size():
    """Radical | radical Schmidt spectrum of a full 221,184-dim state against NumPy's SVD."""
    from rpm_b200 import entanglement as ent
    from rpm_b200 import synthetic

    full = synthetic.full_system()
    v = synthetic.random_phase_vectors(full.dimensions, 1, 9)[0]
    rng = np.random.default_rng(3)
    v = v + 0.05 * (rng.normal(size=v.size) + 1j * rng.normal(size=v.size)) / math.sqrt(v.size)
    left = full.left_axes
    ref = oracle.pure_log_negativity(v, full.dimensions, left)
    assert ent.pure_log_negativity(v, full.dimensions, left) == pytest.approx(ref, abs=1e-9)


@pytest.mark.gpu
def test_gpu_entanglement_cell_prefix_matches_reference():
    import rpm_b200 as rb
    from rpm_b200 import entanglement as ent
    from rpm_b200 import production as p

    dims = tuple(GOLDEN["cell_dims"])
    nuclei = p.selected_nuclei(4)
    h = p.build_hamiltonian(90.0, 0.05, nuclei=nuclei, radicals=p.selected_radicals(4))
    init = p.product_basis_initial_state(dims, p.paired_product_indices(4, p.full_product_basis_indices(20260731, 1)))
    times = GOLDEN["cell_times"]
    res = p.make_propagator(h).propagate(init, times, lambda s: rb.singlet_population(s, dims), store_states=True)
    np.testing.assert_allclose(res.observable_values, GOLDEN["cell_singlet"], atol=1e-11)
    np.testing.assert_allclose(ent.pure_log_negativity(res.states, dims, (0, 2, 3)), GOLDEN["cell_radical_lneg"],
                               atol=1e-9)
    np.testing.assert_allclose(ent.pure_log_negativity(res.states, dims, (0, 1)), GOLDEN["cell_electron_lneg"],
                               atol=1e-9)
    np.testing.assert_allclose(ent.reduced_electron_density(res.states, dims), GOLDEN["cell_rho"], atol=1e-11)
