"""The reference's reduced non-factorizable validation on the CUDA plain FP64 path
(GPU): the adaptive Krylov propagation within 1e-8 of dense propagation for the
eight seeded samples, as tests/test_statevector_baseline.py:396-401 requires of
the reference's own propagator."""

import numpy as np
import pytest

import oracle
from reduced_system import DIMENSIONS, KNOBS, TIMES, dense_populations, sample_state, terms

pytestmark = pytest.mark.gpu


def test_gpu_krylov_matches_dense_for_the_seeded_samples():
    import rpm_b200 as rb

    h = rb.MatrixFreeHamiltonian(DIMENSIONS, terms(rb.LocalTerm))
    dense = oracle.MatrixFreeHamiltonian(DIMENSIONS, terms(oracle.LocalTerm)).explicit_matrix()
    worst = 0.0
    for sample in range(8):
        psi = sample_state(sample)
        res = rb.AdaptiveLanczosPropagator(h, **KNOBS).propagate(psi, TIMES, rb.SingletPopulationObservable(DIMENSIONS))
        worst = max(worst, float(np.max(np.abs(np.asarray(res.observable_values) - dense_populations(dense, psi)))))
    assert worst < 1e-8
