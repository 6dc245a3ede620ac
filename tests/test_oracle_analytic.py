"""The oracle against the reference's closed-form yields (CPU).

* ``truncated_singlet_yield_dense`` generalises poster_reproduction/core.py:455-473
  (dense_truncated_singlet_yield, four levels, singlet start) to any initial
  state: in the four-level case both agree to rounding, and on the production
  0.00125-us grid the Simpson yield of exact populations agrees with the closed
  form well below the coarse-grid quadrature estimate, the reference's own
  validation of that grid.
* ``ensemble_singlet_yield_lorentzian`` restates
  rpm_three_nitrogen_quadrupole.py:100-113: the infinite-horizon yield of the
  singlet (x) maximally mixed nuclear ensemble equals the average of the
  closed-form yields of the nuclear basis states.
"""

import math

import numpy as np
import pytest

import oracle

TAU = 1.0


def _four_level(seed):
    sx, sy, sz = oracle.spin_operators(0.5)
    eye = np.eye(2)
    rng = np.random.default_rng(seed)
    b1, b2 = 0.5 * rng.normal(size=3), 0.5 * rng.normal(size=3)  # local fields, mT
    g = oracle.TWOPI * oracle.GAMMA_E_MHZ_PER_MT
    h = g * (np.kron(b1[0] * sx + b1[1] * sy + b1[2] * sz, eye) + np.kron(eye, b2[0] * sx + b2[1] * sy + b2[2] * sz))
    h = h + oracle.TWOPI * oracle.efimova_hore_electron_coupling_operator(0.05 * 28.0, -0.4 * 28.0,
                                                                          np.array([0.0, 0.0, 1.0]))
    return 0.5 * (h + h.conj().T)


def _small_dense():
    from rpm_b200 import synthetic

    sm = synthetic.small_system()
    h = oracle.MatrixFreeHamiltonian(sm.dimensions, [oracle.LocalTerm(t.axes, t.operator) for t in sm.terms(0.4, 0.0)])
    return sm, h.explicit_matrix()


def _exact_populations(h, dims, psi, times):
    e, v = np.linalg.eigh(h)
    c = v.conj().T @ psi
    return np.array([oracle.singlet_population(v @ (np.exp(-1j * e * t) * c), dims) for t in times])


def _simpson_and_estimate(times, pops):
    fine = oracle.integrate_yield(times, pops, TAU)
    idx = oracle.coarse_grid_indices(times.size)
    return fine, abs(fine - oracle.integrate_yield(times[idx], pops[idx], TAU))


@pytest.mark.parametrize("seed", [3, 8])
def test_four_level_closed_form_is_the_reference_formula(seed):
    h = _four_level(seed)
    singlet = np.array([0.0, 1.0, -1.0, 0.0], dtype=complex) / math.sqrt(2.0)
    got = oracle.truncated_singlet_yield_dense(h, (2, 2), singlet, TAU, 5.0)
    # CORE:455-473 written out for the four-level singlet start
    e, v = np.linalg.eigh(h)
    w = np.abs(v.conj().T @ singlet) ** 2
    decay = 1.0 / TAU + 1j * (e[:, None] - e[None, :])
    ref = float(np.sum(w[:, None] * w[None, :] * (1.0 / TAU) * (1.0 - np.exp(-decay * 5.0)) / decay).real)
    assert abs(got - ref) < 1e-14
    times = oracle.time_grid_us(5.0)
    fine, estimate = _simpson_and_estimate(times, _exact_populations(h, (2, 2), singlet, times))
    assert abs(fine - got) < 0.2 * estimate


def test_random_phase_closed_form_below_the_quadrature_estimate():
    from rpm_b200 import synthetic

    sm, h = _small_dense()
    psi = synthetic.random_phase_vectors(sm.dimensions, 1, 5)[0]
    got = oracle.truncated_singlet_yield_dense(h, sm.dimensions, psi, TAU, 5.0)
    times = oracle.time_grid_us(5.0)
    fine, estimate = _simpson_and_estimate(times, _exact_populations(h, sm.dimensions, psi, times))
    assert abs(fine - got) < 0.2 * estimate


def test_lorentzian_ensemble_is_the_average_over_nuclear_basis_states():
    sm, h = _small_dense()
    dims = sm.dimensions
    n = math.prod(dims)
    m = n // 4
    total = 0.0
    for k in range(m):
        psi = np.zeros(n, dtype=complex)
        psi[m + k], psi[2 * m + k] = 1.0 / math.sqrt(2.0), -1.0 / math.sqrt(2.0)
        total += oracle.truncated_singlet_yield_dense(h, dims, psi, TAU, 40.0)  # exp(-40) truncation
    assert abs(oracle.ensemble_singlet_yield_lorentzian(h, dims, TAU) - total / m) < 1e-13
