"""The reference's reduced non-factorizable validation against the oracle (CPU):
exact density-matrix trace = exhaustive nuclear-basis average (1e-12), the
adaptive Krylov propagation within 1e-8 of dense propagation for the eight
seeded samples, and the 256-sample random-phase average within 1e-2 rms.
"""

import numpy as np
from scipy.linalg import expm

import oracle
from reduced_system import DIMENSIONS, KNOBS, NUCLEAR, SEED, SINGLET, TIMES, dense_populations, sample_state, terms


def _dense():
    return oracle.MatrixFreeHamiltonian(DIMENSIONS, terms(oracle.LocalTerm)).explicit_matrix()


def test_exact_trace_equals_exhaustive_basis_average():
    dense = _dense()
    proj = np.kron(np.outer(SINGLET, SINGLET.conj()), np.eye(NUCLEAR))
    rho0 = np.kron(np.outer(SINGLET, SINGLET.conj()), np.eye(NUCLEAR) / NUCLEAR)
    worst = 0.0
    for t in TIMES:
        u = expm(-1j * dense * t)
        exact = float(np.trace(proj @ u @ rho0 @ u.conj().T).real)
        basis = np.mean([float(np.vdot(u @ np.kron(SINGLET, np.eye(NUCLEAR)[:, k]),
                                       proj @ (u @ np.kron(SINGLET, np.eye(NUCLEAR)[:, k]))).real)
                         for k in range(NUCLEAR)])
        worst = max(worst, abs(exact - basis))
    assert worst < 1e-12


def test_oracle_krylov_matches_dense_for_the_seeded_samples():
    h = oracle.MatrixFreeHamiltonian(DIMENSIONS, terms(oracle.LocalTerm))
    dense = h.explicit_matrix()
    worst = 0.0
    for sample in range(8):
        psi = sample_state(sample)
        res = oracle.AdaptiveLanczosPropagator(h, **KNOBS).propagate(
            psi, TIMES, lambda v: oracle.singlet_population(v, DIMENSIONS))
        worst = max(worst, float(np.max(np.abs(np.asarray(res.observable_values) - dense_populations(dense, psi)))))
    assert worst < 1e-8


def test_random_phase_average_converges_to_the_exact_trace():
    dense = _dense()
    proj = np.kron(np.outer(SINGLET, SINGLET.conj()), np.eye(NUCLEAR))
    rho0 = np.kron(np.outer(SINGLET, SINGLET.conj()), np.eye(NUCLEAR) / NUCLEAR)
    units = [expm(-1j * dense * t) for t in TIMES]
    exact = np.array([float(np.trace(proj @ u @ rho0 @ u.conj().T).real) for u in units])
    rng = np.random.default_rng(SEED)
    traces = []
    for _ in range(256):
        psi = np.kron(SINGLET, np.exp(1j * rng.uniform(0.0, oracle.TWOPI, NUCLEAR)) / np.sqrt(NUCLEAR))
        traces.append([float(np.vdot(u @ psi, proj @ (u @ psi)).real) for u in units])
    mean = np.asarray(traces).mean(axis=0)
    assert float(np.sqrt(np.mean((mean - exact) ** 2))) < 1e-2
