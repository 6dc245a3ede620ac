"""The reduced non-factorizable J + D + Q system of the reference's validation
(rpm_quantum_needle_validation.py:730-817, reduced_validation; its test
tests/test_statevector_baseline.py:396-401): dims (2, 2, 3, 2), field 50 uT
at 67 degrees, one hyperfine tensor per radical, a full electron-electron
tensor with exchange, and a spin-1 quadrupole; observation grid 0..2 us in
41 points; Krylov knobs 8-24 (+4), embedded offset 2, budget 1e-10, steps
0.25 us; samples seeded by SeedSequence([9917, sample]).
"""

import math

import numpy as np

import oracle

DIMENSIONS = (2, 2, 3, 2)
SEED = 9917
KNOBS = dict(minimum_dimension=8, maximum_dimension=24, dimension_increment=4, embedded_offset=2,
             state_error_budget=1e-10, initial_step_us=0.25, maximum_step_us=0.25)
TIMES = np.linspace(0.0, 2.0, 41)
SINGLET = np.array([0.0, 1.0, -1.0, 0.0], dtype=complex) / math.sqrt(2.0)
NUCLEAR = 6


def terms(local_term):
    """(axes, operator, label) terms built with ``local_term`` (the oracle's or rpm_b200's LocalTerm)."""
    sx, sy, sz = oracle.spin_operators(0.5)
    b = oracle.field_vector_mT(67.0, 50.0)
    zeeman = oracle.TWOPI * oracle.GAMMA_E_MHZ_PER_MT * (b[0] * sx + b[1] * sy + b[2] * sz)
    hf_a = oracle.TWOPI * np.array([[0.15, 0.02, 0.01], [0.02, -0.08, 0.03], [0.01, 0.03, 1.2]])
    hf_b = oracle.TWOPI * np.array([[0.2, -0.03, 0.01], [-0.03, 0.1, 0.02], [0.01, 0.02, 0.8]])
    ee = oracle.TWOPI * (np.array([[0.12, 0.03, -0.02], [0.03, -0.07, 0.04], [-0.02, 0.04, -0.05]]) - 0.5 * np.eye(3))
    q = oracle.TWOPI * np.diag([-0.025, -0.025, 0.05])
    return [
        local_term((0,), zeeman, "eA Zeeman"),
        local_term((1,), zeeman, "eB Zeeman"),
        local_term((0, 2), oracle.two_spin_coupling_operator(0.5, 1.0, hf_a), "A hyperfine"),
        local_term((1, 3), oracle.two_spin_coupling_operator(0.5, 0.5, hf_b), "B hyperfine"),
        local_term((0, 1), oracle.two_spin_coupling_operator(0.5, 0.5, ee), "nonfactorizable J+D"),
        local_term((2,), oracle.quadrupole_operator(1.0, q), "spin-1 quadrupole"),
    ]


def sample_state(sample: int) -> np.ndarray:
    seed = int(np.random.SeedSequence([SEED, int(sample)]).generate_state(1, dtype=np.uint32)[0])
    rng = np.random.default_rng(seed)
    nuclear = np.exp(1.0j * rng.uniform(0.0, oracle.TWOPI, NUCLEAR)) / math.sqrt(NUCLEAR)
    return np.kron(SINGLET, nuclear)


def dense_populations(dense, state) -> np.ndarray:
    from scipy.linalg import expm

    out = np.empty(TIMES.size)
    for k, t in enumerate(TIMES):
        psi = expm(-1j * dense * t) @ state
        out[k] = oracle.singlet_population(psi, DIMENSIONS)
    return out
