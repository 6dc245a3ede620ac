"""The CUDA path against the reference's closed-form yields (GPU).

The closed forms (oracle ``truncated_singlet_yield_dense``, restating
poster_reproduction/core.py:455-473 for any initial state) are exact
integrals; the CUDA path integrates populations on the production
0.00125-us grid by Simpson's rule (JD:418-420).  Bars: the plain FP64 path's
yield within a fifth of its own coarse-grid quadrature estimate of the closed
form (the reference's validation of that grid); the batched mixed-precision
path's basis-state ensemble within 1e-6 of the closed forms.
"""

import math

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

TAU = 1.0
HORIZON = 5.0


def _small():
    from rpm_b200 import synthetic

    sm = synthetic.small_system()
    terms = sm.terms(0.4, 0.0)
    dense = oracle.MatrixFreeHamiltonian(sm.dimensions, [oracle.LocalTerm(t.axes, t.operator) for t in terms])
    return sm, terms, dense.explicit_matrix()


def test_plain_fp64_yield_meets_the_closed_form():
    import rpm_b200 as rb
    from rpm_b200 import synthetic

    sm, terms, hd = _small()
    h = rb.MatrixFreeHamiltonian(sm.dimensions, terms)
    times = oracle.time_grid_us(HORIZON)
    idx = oracle.coarse_grid_indices(times.size)
    for seed in (5, 6):
        psi = synthetic.random_phase_vectors(sm.dimensions, 1, seed)[0]
        res = rb.AdaptiveLanczosPropagator(h, state_error_budget=1e-10).propagate(
            psi, times, rb.SingletPopulationObservable(sm.dimensions))
        pops = np.asarray(res.observable_values)
        fine = rb.integrate_yield(times, pops, TAU)
        estimate = abs(fine - rb.integrate_yield(times[idx], pops[idx], TAU))
        closed = oracle.truncated_singlet_yield_dense(hd, sm.dimensions, psi, TAU, HORIZON)
        assert abs(fine - closed) < 0.2 * estimate + 1e-9, (fine, closed, estimate)


def test_batched_basis_state_ensemble_meets_the_closed_forms():
    import rpm_b200 as rb
    from rpm_b200.batched import BatchedPropagator

    sm, terms, hd = _small()
    dims = sm.dimensions
    n = math.prod(dims)
    m = n // 4
    states = []
    for k in range(m):
        psi = np.zeros(n, dtype=complex)
        psi[m + k], psi[2 * m + k] = 1.0 / math.sqrt(2.0), -1.0 / math.sqrt(2.0)
        states.append(psi)
    h = rb.CompiledFullPairHamiltonian(dims, terms, left_axes=sm.left_axes, right_axes=sm.right_axes)
    times = oracle.time_grid_us(HORIZON)
    out = BatchedPropagator([h], krylov_dimension=30, state_error_budget=1e-9).propagate(states, times,
                                                                                         lifetime_us=TAU)
    closed = np.array([oracle.truncated_singlet_yield_dense(hd, dims, s, TAU, HORIZON) for s in states])
    assert np.max(np.abs(out.yields - closed)) < 1e-6
    assert abs(out.yields.mean() - closed.mean()) < 1e-6
