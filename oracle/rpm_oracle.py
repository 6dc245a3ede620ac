"""NumPy restatement of the reference's FP64 radical-pair hot path (oracle).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Every function names the reference file and lines whose behaviour it restates.
Paths are relative to ``Realistic system size/code/`` of sam-not-smart/RPM:

* ``ENG``  = ``rpm_statevector_engine.py``
* ``MOD``  = ``rpm_quantum_needle_model.py``
* ``CORE`` = ``poster_reproduction/core.py``
* ``JD``   = ``rpm_quantum_needle_jd_sweeps.py``

Arithmetic is complex128 / float64 throughout, as in the reference.  The
small tridiagonal eigenproblem uses ``numpy.linalg.eigh`` on the assembled
symmetric tridiagonal (the reference calls LAPACK through
``scipy.linalg.eigh_tridiagonal``); Simpson's rule is restated in NumPy with
the same non-uniform and even-count (Cartwright) formulas that
``scipy.integrate.simpson`` 1.18 applies.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Iterable, Sequence

import numpy as np

TWOPI = 2.0 * math.pi
GAMMA_E_MHZ_PER_MT = 28.0  # MOD:17


# ---------------------------------------------------------------------------
# Spin algebra and local operators
# ---------------------------------------------------------------------------

def spin_operators(spin: float) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(Sx, Sy, Sz) in the descending-m basis m = I, I-1, ..., -I (MOD:178-192)."""
    d = int(round(2.0 * spin + 1.0))
    m = spin - np.arange(d, dtype=float)
    # <m+1| I+ |m> = sqrt(I(I+1) - m(m+1)); I+ sits on the first superdiagonal
    up = np.zeros((d, d), dtype=complex)
    for k in range(1, d):
        up[k - 1, k] = math.sqrt(spin * (spin + 1.0) - m[k] * (m[k] + 1.0))
    down = up.conj().T
    return (up + down) / 2.0, (up - down) / 2.0j, np.diag(m).astype(complex)


def field_vector_mT(theta_deg: float, field_microT: float = 50.0) -> np.ndarray:
    """Field in the molecular zx plane, in mT (MOD:195-199)."""
    th = np.deg2rad(theta_deg)
    return 1e-3 * field_microT * np.array([np.sin(th), 0.0, np.cos(th)])


def two_spin_coupling_operator(left_spin: float, right_spin: float, tensor) -> np.ndarray:
    """sum_ab T_ab S_a (x) I_b (ENG:269-287)."""
    t = np.asarray(tensor, dtype=float)
    if t.shape != (3, 3):
        raise ValueError("A two-spin coupling tensor must be 3x3.")
    s = spin_operators(left_spin)
    i = spin_operators(right_spin)
    out = np.zeros((s[0].shape[0] * i[0].shape[0],) * 2, dtype=complex)
    for a in range(3):
        for b in range(3):
            if t[a, b] != 0.0:
                out += t[a, b] * np.kron(s[a], i[b])
    return out


def quadrupole_operator(spin: float, tensor) -> np.ndarray:
    """sum_ab Q_ab {I_a, I_b}/2 (ENG:332-349)."""
    q = np.asarray(tensor, dtype=float)
    if q.shape != (3, 3):
        raise ValueError("A quadrupole tensor must be 3x3.")
    if not np.allclose(q, q.T, atol=1e-14, rtol=0.0):
        raise ValueError("A quadrupole tensor must be symmetric.")
    ops = spin_operators(spin)
    out = np.zeros_like(ops[0])
    for a in range(3):
        for b in range(3):
            if q[a, b] != 0.0:
                out += 0.5 * q[a, b] * (ops[a] @ ops[b] + ops[b] @ ops[a])
    return out


def efimova_hore_electron_coupling_operator(exchange_J_MHz, dipolar_D_MHz, dipolar_axis) -> np.ndarray:
    """-J(S^2 - 1) + D((S.n)^2 - S^2/3) on the two electrons, in MHz (ENG:290-329)."""
    n = np.asarray(dipolar_axis, dtype=float)
    if n.shape != (3,):
        raise ValueError("dipolar_axis must be a length-3 vector.")
    nn = float(np.linalg.norm(n))
    if nn == 0.0:
        raise ValueError("dipolar_axis must be nonzero.")
    n = n / nn
    s = spin_operators(0.5)
    e2 = np.eye(2, dtype=complex)
    total = [np.kron(op, e2) + np.kron(e2, op) for op in s]
    s2 = sum(op @ op for op in total)
    sn = sum(c * op for c, op in zip(n, total))
    h = -float(exchange_J_MHz) * (s2 - np.eye(4)) + float(dipolar_D_MHz) * (sn @ sn - s2 / 3.0)
    return 0.5 * (h + h.conj().T)


# ---------------------------------------------------------------------------
# Physical model tables (MOD:37-131).  Hyperfine tensors in mT.
# ---------------------------------------------------------------------------

@dataclass(frozen=True)
class Nucleus:
    name: str
    spin: float
    tensor_mT: np.ndarray = field(compare=False)

    @property
    def dimension(self) -> int:
        return int(round(2.0 * self.spin + 1.0))


def _sym(rows):
    return np.array(rows, dtype=float)


FAD_NUCLEI = (
    Nucleus("N5", 1.0, _sym([[-0.0989, 0.0039, 0.0], [0.0039, -0.0881, 0.0], [0.0, 0.0, 1.7569]])),
    Nucleus("N10", 1.0, _sym([[-0.0190, -0.0048, 0.0], [-0.0048, -0.0196, 0.0], [0.0, 0.0, 0.6046]])),
    Nucleus("H6", 0.5, _sym([[-0.2569, -0.1273, 0.0], [-0.1273, -0.4711, 0.0], [0.0, 0.0, -0.4336]])),
    Nucleus("H8a", 0.5, 0.4399 * np.eye(3)),
    Nucleus("H8b", 0.5, 0.4399 * np.eye(3)),
    Nucleus("H8c", 0.5, 0.4399 * np.eye(3)),
    Nucleus("Hbeta", 0.5, 0.4070 * np.eye(3)),
)
TRP_NUCLEI = (
    Nucleus("N1", 1.0, _sym([[-0.0336, 0.0924, -0.1354], [0.0924, 0.3303, -0.5318], [-0.1354, -0.5318, 0.6680]])),
    Nucleus("H1", 0.5, _sym([[-0.9920, -0.2091, -0.2003], [-0.2091, -0.2631, 0.2803], [-0.2003, 0.2803, -0.5398]])),
    Nucleus("H2", 0.5, _sym([[-0.2843, 0.1757, 0.1525], [0.1757, -0.2798, 0.0975], [0.1525, 0.0975, -0.2699]])),
    Nucleus("H4", 0.5, _sym([[-0.5596, -0.1956, -0.1657], [-0.1956, -0.4020, 0.0762], [-0.1657, 0.0762, -0.5021]])),
    Nucleus("H5", 0.5, _sym([[0.0051, 0.0616, 0.0694], [0.0616, -0.0665, 0.0391], [0.0694, 0.0391, -0.0586]])),
    Nucleus("H7", 0.5, _sym([[-0.4355, -0.1541, -0.1239], [-0.1541, -0.2777, 0.0864], [-0.1239, 0.0864, -0.3770]])),
    Nucleus("Hbeta1", 0.5, _sym([[1.5808, -0.0453, -0.0506], [-0.0453, 1.5575, 0.0988], [-0.0506, 0.0988, 1.6752]])),
)
ALL_NUCLEI = FAD_NUCLEI + TRP_NUCLEI
NUCLEAR_RADICALS = ("FAD",) * len(FAD_NUCLEI) + ("TrpH",) * len(TRP_NUCLEI)
SYSTEM_DIMENSIONS = (2, 2) + tuple(n.dimension for n in ALL_NUCLEI)


def _quadrupole_in_hyperfine_frame(hf, principal, orientation):
    """Traceless Q placed on the hyperfine principal axes (MOD:69-102)."""
    p = np.asarray(principal, dtype=float)
    p = p - p.mean()
    w, axes = np.linalg.eigh(hf)
    normal = int(np.argmax(np.abs(w)))
    plane = [k for k in range(3) if k != normal]
    diag = np.empty(3)
    if orientation == "ring_normal":
        diag[normal], diag[plane[0]], diag[plane[1]] = p[2], p[0], p[1]
    elif orientation == "ring_plane_provisional":
        diag[plane[0]], diag[plane[1]], diag[normal] = p[2], p[0], p[1]
    else:
        raise ValueError(orientation)
    q = axes @ np.diag(diag) @ axes.T
    return 0.5 * (q + q.T)


QUADRUPOLE_TENSORS_MT = {
    "FAD:N5": _quadrupole_in_hyperfine_frame(FAD_NUCLEI[0].tensor_mT, (0.031, 0.041, -0.072), "ring_plane_provisional"),
    "FAD:N10": _quadrupole_in_hyperfine_frame(FAD_NUCLEI[1].tensor_mT, (0.032, 0.041, -0.072), "ring_normal"),
    "TrpH:N1": _quadrupole_in_hyperfine_frame(TRP_NUCLEI[0].tensor_mT, (0.016, 0.020, -0.036), "ring_normal"),
}

# JD:81 and JD:101-102: D = -2783/8 uT, equivalent-field uT -> MHz at 28 MHz/mT
R2_D_PAPER_UT = -2783.0 / 8.0


def uT_to_MHz(value_uT: float) -> float:
    return float(value_uT) * GAMMA_E_MHZ_PER_MT / 1000.0


# ---------------------------------------------------------------------------
# Matrix-free Hamiltonians
# ---------------------------------------------------------------------------

@dataclass(frozen=True)
class LocalTerm:
    """(axes, d x d operator, label) -- ENG:28-34."""
    axes: tuple
    operator: np.ndarray = field(compare=False)
    label: str = ""


class MatrixFreeHamiltonian:
    """Sum of local terms applied mode by mode (ENG:46-129)."""

    def __init__(self, dimensions: Iterable[int], terms: Iterable[LocalTerm], *, hermitian_tolerance=1e-12):
        self.dimensions = tuple(int(v) for v in dimensions)
        if not self.dimensions or min(self.dimensions) < 1:
            raise ValueError("Every tensor dimension must be positive.")
        self.dimension = math.prod(self.dimensions)
        self.shape = (self.dimension, self.dimension)
        self.dtype = np.dtype(np.complex128)
        self.matvec_count = 0
        checked = []
        for term in terms:
            axes = tuple(int(a) for a in term.axes)
            if not axes or len(set(axes)) != len(axes):
                raise ValueError("Local term must have unique active axes.")
            if min(axes) < 0 or max(axes) >= len(self.dimensions):
                raise ValueError("Local term contains an out-of-range axis.")
            d = math.prod(self.dimensions[a] for a in axes)
            op = np.asarray(term.operator, dtype=complex)
            if op.shape != (d, d):
                raise ValueError(f"Local term has shape {op.shape}; expected {(d, d)}.")
            if np.linalg.norm(op - op.conj().T) > hermitian_tolerance * max(1.0, float(np.linalg.norm(op))):
                raise ValueError("Local term is not Hermitian.")
            checked.append(LocalTerm(axes, np.ascontiguousarray(op), term.label))
        self.terms = tuple(checked)

    def _apply(self, tensor: np.ndarray) -> np.ndarray:
        out = np.zeros_like(tensor)
        for term in self.terms:
            k = len(term.axes)
            active = tuple(self.dimensions[a] for a in term.axes)
            # bring the active axes to the front, contract, put them back
            front = np.moveaxis(tensor, term.axes, tuple(range(k)))
            rest = front.shape[k:]
            applied = (term.operator @ front.reshape(math.prod(active), -1)).reshape(active + rest)
            out += np.moveaxis(applied, tuple(range(k)), term.axes)
        return out

    def matvec(self, vector) -> np.ndarray:
        flat = np.asarray(vector, dtype=complex).reshape(-1)
        if flat.size != self.dimension:
            raise ValueError(f"Vector length {flat.size} does not match {self.dimension}.")
        result = self._apply(flat.reshape(self.dimensions)).reshape(-1)
        self.matvec_count += 1
        return result

    def matmat(self, matrix) -> np.ndarray:
        m = np.asarray(matrix, dtype=complex)
        if m.ndim != 2 or m.shape[0] != self.dimension:
            raise ValueError(f"Matrix must have shape ({self.dimension}, n_vectors).")
        return np.stack([self.matvec(m[:, j]) for j in range(m.shape[1])], axis=1)

    def explicit_matrix(self) -> np.ndarray:
        return self.matmat(np.eye(self.dimension, dtype=complex))


class CompiledFullPairHamiltonian:
    """Radical-split action L.Psi + Psi.R^T + electron-pair term (ENG:132-266).

    The two radical blocks are held dense here (576 and 384 wide at full size),
    which is exact and fast enough for an oracle.
    """

    def __init__(self, dimensions, terms, *, left_axes, right_axes, electron_pair_axes=(0, 1)):
        src = MatrixFreeHamiltonian(dimensions, terms)
        self.dimensions, self.dimension, self.shape = src.dimensions, src.dimension, src.shape
        self.dtype, self.terms, self.matvec_count = src.dtype, src.terms, 0
        left, right = tuple(int(a) for a in left_axes), tuple(int(a) for a in right_axes)
        if not left or not right or set(left) & set(right):
            raise ValueError("Full-pair axis groups must be nonempty and disjoint.")
        if set(left + right) != set(range(len(self.dimensions))):
            raise ValueError("Full-pair axis groups must partition every tensor axis.")
        if left[0] != electron_pair_axes[0] or right[0] != electron_pair_axes[1]:
            raise ValueError("Each radical electron must be first in its axis group.")
        if self.dimensions[left[0]] != 2 or self.dimensions[right[0]] != 2:
            raise ValueError("The electron-pair axes must both have dimension two.")
        lpos = {a: i for i, a in enumerate(left)}
        rpos = {a: i for i, a in enumerate(right)}
        lterms, rterms = [], []
        pair = np.zeros((4, 4), dtype=complex)
        for t in self.terms:
            if all(a in lpos for a in t.axes):
                lterms.append(LocalTerm(tuple(lpos[a] for a in t.axes), t.operator, t.label))
            elif all(a in rpos for a in t.axes):
                rterms.append(LocalTerm(tuple(rpos[a] for a in t.axes), t.operator, t.label))
            elif tuple(t.axes) == tuple(electron_pair_axes):
                pair += t.operator
            else:
                raise ValueError("Cross-radical terms must act on the configured electron pair.")
        self.left_axes, self.right_axes = left, right
        self.permutation = left + right
        self.inverse_permutation = tuple(int(v) for v in np.argsort(self.permutation))
        self.left_dimensions = tuple(self.dimensions[a] for a in left)
        self.right_dimensions = tuple(self.dimensions[a] for a in right)
        self.left_dimension = math.prod(self.left_dimensions)
        self.right_dimension = math.prod(self.right_dimensions)
        # dense blocks assembled term by term, then held as CSR like the
        # reference (scipy.sparse.csr_matrix + eliminate_zeros)
        import scipy.sparse

        left_dense = MatrixFreeHamiltonian(self.left_dimensions, lterms).explicit_matrix()
        right_dense = MatrixFreeHamiltonian(self.right_dimensions, rterms).explicit_matrix()
        self.left_operator = scipy.sparse.csr_matrix(left_dense)
        self.right_operator = scipy.sparse.csr_matrix(right_dense)
        self.left_operator.eliminate_zeros()
        self.right_operator.eliminate_zeros()
        self.electron_pair_operator = pair.reshape(2, 2, 2, 2)

    def matvec(self, vector) -> np.ndarray:
        flat = np.asarray(vector, dtype=complex).reshape(-1)
        if flat.size != self.dimension:
            raise ValueError(f"Vector length {flat.size} does not match {self.dimension}.")
        grouped = np.transpose(flat.reshape(self.dimensions), self.permutation)
        psi = grouped.reshape(self.left_dimension, self.right_dimension)
        out = self.left_operator @ psi + (self.right_operator @ psi.T).T
        four = grouped.reshape(2, self.left_dimension // 2, 2, self.right_dimension // 2)
        out += np.einsum("abcd,cxdy->axby", self.electron_pair_operator, four, optimize=True).reshape(psi.shape)
        back = np.transpose(out.reshape(self.left_dimensions + self.right_dimensions), self.inverse_permutation)
        self.matvec_count += 1
        return back.reshape(-1)

    def matmat(self, matrix) -> np.ndarray:
        m = np.asarray(matrix, dtype=complex)
        if m.ndim != 2 or m.shape[0] != self.dimension:
            raise ValueError(f"Matrix must have shape ({self.dimension}, n_vectors).")
        return np.stack([self.matvec(m[:, j]) for j in range(m.shape[1])], axis=1)

    def explicit_matrix(self) -> np.ndarray:
        return self.matmat(np.eye(self.dimension, dtype=complex))


# ---------------------------------------------------------------------------
# Production and quantum-needle assembly
# ---------------------------------------------------------------------------

def _zeeman(theta_deg, field_microT):
    s = spin_operators(0.5)
    b = field_vector_mT(theta_deg, field_microT)
    return TWOPI * GAMMA_E_MHZ_PER_MT * sum(c * op for c, op in zip(b, s))


def build_hamiltonian(theta_deg, field_mT, *, nuclei=ALL_NUCLEI, radicals=NUCLEAR_RADICALS,
                      quadrupole_scale=1.0, exchange_J_uT=0.0, d_paper_uT=0.0,
                      dipolar_axis=(1.0, 0.0, 0.0), hyperfine_overrides_mT=None):
    """Term list and radical split of CORE:172-229 (Efimova-Hore J/D, CORE:154-161).

    Returns a ``CompiledFullPairHamiltonian`` like the reference.
    """
    dims = (2, 2) + tuple(n.dimension for n in nuclei)
    z = _zeeman(theta_deg, float(field_mT) * 1000.0)
    terms = [LocalTerm((0,), z, "electron A Zeeman"), LocalTerm((1,), z, "electron B Zeeman")]
    overrides = hyperfine_overrides_mT or {}
    for k, (nuc, rad) in enumerate(zip(nuclei, radicals)):
        key = f"{rad}:{nuc.name}"
        tensor = np.asarray(overrides.get(key, nuc.tensor_mT), dtype=float)
        e = 0 if rad == "FAD" else 1
        terms.append(LocalTerm((e, k + 2), TWOPI * GAMMA_E_MHZ_PER_MT * two_spin_coupling_operator(0.5, nuc.spin, tensor),
                               f"{key} hyperfine"))
        q = QUADRUPOLE_TENSORS_MT.get(key)
        if q is not None and quadrupole_scale != 0.0:
            terms.append(LocalTerm((k + 2,), quadrupole_operator(nuc.spin, TWOPI * GAMMA_E_MHZ_PER_MT * quadrupole_scale * q),
                                   f"{key} quadrupole"))
    terms.append(LocalTerm((0, 1), TWOPI * efimova_hore_electron_coupling_operator(
        uT_to_MHz(exchange_J_uT), uT_to_MHz(d_paper_uT), np.asarray(dipolar_axis, dtype=float)),
        "Efimova-Hore exchange + full nonsecular dipolar"))
    left = (0,) + tuple(k + 2 for k, r in enumerate(radicals) if r == "FAD")
    right = (1,) + tuple(k + 2 for k, r in enumerate(radicals) if r == "TrpH")
    return CompiledFullPairHamiltonian(dims, terms, left_axes=left, right_axes=right)


# ---------------------------------------------------------------------------
# Initial states and observables
# ---------------------------------------------------------------------------

SINGLET = np.array([0.0, 1.0, -1.0, 0.0], dtype=complex) / math.sqrt(2.0)


def production_sample_seed(base: int, sample_id: int) -> int:
    """SeedSequence([base, 0xA11CE, sample]) -> first uint32 word (JD:373-375)."""
    return int(np.random.SeedSequence([int(base), 0xA11CE, int(sample_id)]).generate_state(1, dtype=np.uint32)[0])


def random_phase_nuclear_state(nuclear_dimension: int, rng: np.random.Generator) -> np.ndarray:
    """e^{i phi}/sqrt(M), phi ~ U[0, 2 pi) (ENG:472-477)."""
    phases = rng.uniform(0.0, TWOPI, int(nuclear_dimension))
    return np.exp(1.0j * phases) / math.sqrt(nuclear_dimension)


def singlet_initial_state(dimensions, rng) -> np.ndarray:
    """Electron singlet (x) random-phase nuclei (ENG:480-489)."""
    dims = tuple(int(v) for v in dimensions)
    if dims[:2] != (2, 2):
        raise ValueError("The first two axes must be the two electron spins.")
    return np.kron(SINGLET, random_phase_nuclear_state(math.prod(dims[2:]), rng))


def random_phase_initial_state(dimensions, master_seed: int, sample_id: int) -> np.ndarray:
    """CORE:250-258."""
    rng = np.random.default_rng(production_sample_seed(master_seed, sample_id))
    return singlet_initial_state(dimensions, rng)


def singlet_population(vector, dimensions) -> float:
    """|| (psi[0,1,:] - psi[1,0,:]) / sqrt 2 ||^2 (ENG:492-497)."""
    e = np.asarray(vector, dtype=complex).reshape(2, 2, -1)
    amp = (e[0, 1] - e[1, 0]) / math.sqrt(2.0)
    return float(np.vdot(amp, amp).real)


class SingletPopulationObservable:
    """Singlet population with the Krylov-basis projection shortcut (ENG:500-538)."""

    def __init__(self, dimensions):
        dims = tuple(int(v) for v in dimensions)
        if dims[:2] != (2, 2):
            raise ValueError("The first two axes must be the two electron spins.")
        self.dimensions = dims

    def __call__(self, vector) -> float:
        return singlet_population(vector, self.dimensions)

    def project_basis(self, basis) -> np.ndarray:
        v = np.asarray(basis, dtype=complex)
        if v.ndim != 2 or v.shape[0] != math.prod(self.dimensions):
            raise ValueError("Krylov basis has the wrong shape.")
        e = v.reshape(2, 2, -1, v.shape[1])
        a = (e[0, 1] - e[1, 0]) / math.sqrt(2.0)
        g = a.conj().T @ a
        return 0.5 * (g + g.conj().T)

    @staticmethod
    def evaluate_projected(projected, coefficients, state_norm) -> float:
        return float(state_norm * state_norm * np.vdot(coefficients, projected @ coefficients).real)


def state_error_to_population_bound(state_error: float) -> float:
    """min(1, 2 eps + eps^2) (ENG:541-543)."""
    e = max(0.0, float(state_error))
    return min(1.0, 2.0 * e + e * e)


# ---------------------------------------------------------------------------
# Adaptive Lanczos propagation (ENG:546-933)
# ---------------------------------------------------------------------------

@dataclass(frozen=True)
class PropagationStats:
    accepted_steps: int
    rejected_steps: int
    matvecs: int
    maximum_krylov_dimension: int
    minimum_step_us: float
    maximum_step_us: float
    accumulated_state_error: float
    maximum_norm_error: float


@dataclass(frozen=True)
class PropagationResult:
    times_us: np.ndarray
    observable_values: np.ndarray
    observable_error_bounds: np.ndarray
    state_error_estimates: np.ndarray
    states: np.ndarray | None
    final_state: np.ndarray
    stats: PropagationStats


class _Spectral:
    """Eigen-decomposition of a symmetric tridiagonal, used for exp(-i T t) e1."""

    def __init__(self, alpha, beta):
        m = len(alpha)
        if m == 1:
            self.w = np.asarray(alpha, dtype=float).copy()
            self.q = np.ones((1, 1))
        else:
            t = np.diag(np.asarray(alpha, dtype=float)) + np.diag(beta, 1) + np.diag(beta, -1)
            self.w, self.q = np.linalg.eigh(t)
        self.q0 = self.q[0, :].copy()

    def coefficients(self, time_us: float) -> np.ndarray:
        return self.q @ (np.exp(-1.0j * self.w * time_us) * self.q0)


def projected_coefficients(alpha, beta, time_us) -> np.ndarray:
    """exp(-i T_m t) e1 (ENG:569-582)."""
    return _Spectral(alpha, beta).coefficients(time_us)


class AdaptiveLanczosPropagator:
    """Step-for-step restatement of the reference controller (ENG:612-933)."""

    def __init__(self, hamiltonian, *, minimum_dimension=24, maximum_dimension=64, dimension_increment=8,
                 embedded_offset=4, safety_factor=2.0, state_error_budget=2.4e-5, initial_step_us=0.05,
                 maximum_step_us=0.25, minimum_step_us=1e-9, breakdown_tolerance=1e-14):
        if minimum_dimension <= embedded_offset:
            raise ValueError("minimum_dimension must exceed embedded_offset.")
        if maximum_dimension < minimum_dimension:
            raise ValueError("maximum_dimension must not be smaller than minimum_dimension.")
        self.hamiltonian = hamiltonian
        self.minimum_dimension, self.maximum_dimension = minimum_dimension, maximum_dimension
        self.dimension_increment, self.embedded_offset = dimension_increment, embedded_offset
        self.safety_factor, self.state_error_budget = safety_factor, state_error_budget
        self.initial_step_us, self.maximum_step_us = initial_step_us, maximum_step_us
        self.minimum_step_us, self.breakdown_tolerance = minimum_step_us, breakdown_tolerance

    def _basis(self, state, target):
        """Hermitian Lanczos with two classical Gram-Schmidt passes (ENG:651-688)."""
        norm = float(np.linalg.norm(state))
        if norm == 0.0:
            raise ValueError("Cannot propagate the zero vector.")
        m = min(int(target), state.size)
        v = np.empty((state.size, m), dtype=complex)
        # rows of vh are the conjugated basis vectors, kept up to date so the
        # projections need no conjugate copy of the block
        vh = np.empty((m, state.size), dtype=complex)
        alpha = np.empty(m)
        beta = np.empty(max(m - 1, 0))
        v[:, 0] = state / norm
        np.conjugate(v[:, 0], out=vh[0])
        size = m
        for j in range(m):
            w = self.hamiltonian.matvec(v[:, j])
            alpha[j] = float(np.vdot(v[:, j], w).real)
            w -= alpha[j] * v[:, j]
            if j:
                w -= beta[j - 1] * v[:, j - 1]
            block, block_h = v[:, : j + 1], vh[: j + 1]
            for _ in range(2):
                w -= block @ (block_h @ w)
            if j == m - 1:
                break
            b = float(np.linalg.norm(w))
            beta[j] = b
            if b <= self.breakdown_tolerance:
                size = j + 1
                break
            v[:, j + 1] = w / b
            np.conjugate(v[:, j + 1], out=vh[j + 1])
        return v[:, :size], alpha[:size], beta[: max(0, size - 1)]

    def _candidate(self, alpha, beta, dimension, time_us, state_norm):
        """Embedded error of dims (d, d - offset) (ENG:690-715)."""
        d = min(dimension, alpha.size)
        high = projected_coefficients(alpha[:d], beta[: max(0, d - 1)], time_us)
        low_d = max(1, d - self.embedded_offset)
        if low_d == d:
            return high, 0.0
        low = projected_coefficients(alpha[:low_d], beta[: max(0, low_d - 1)], time_us)
        diff = high.copy()
        diff[:low_d] -= low
        return high, self.safety_factor * state_norm * float(np.linalg.norm(diff))

    def _ladder(self, start):
        dims = list(range(start, self.maximum_dimension + 1, self.dimension_increment))
        if not dims or dims[-1] != self.maximum_dimension:
            dims.append(self.maximum_dimension)
        return dims

    def propagate(self, initial_state, times_us, observable, *, store_states=False, progress_callback=None):
        times = np.asarray([float(t) for t in times_us], dtype=float)
        if times.ndim != 1 or times.size == 0:
            raise ValueError("At least one observation time is required.")
        if np.any(times < 0.0) or np.any(np.diff(times) <= 0.0):
            raise ValueError("Observation times must be nonnegative and strictly increasing.")
        state = np.asarray(initial_state, dtype=complex).reshape(-1).copy()
        if state.size != self.hamiltonian.dimension:
            raise ValueError("Initial state dimension does not match the Hamiltonian.")
        projected_ok = (not store_states and callable(getattr(observable, "project_basis", None))
                        and callable(getattr(observable, "evaluate_projected", None)))
        n_t = times.size
        values, bounds, serr = np.empty(n_t), np.empty(n_t), np.empty(n_t)
        stored = np.empty((n_t, state.size), dtype=complex) if store_states else None
        cursor, now, acc_err = 0, 0.0, 0.0
        accepted = rejected = max_dim = 0
        used: list[float] = []
        max_norm_err = abs(float(np.linalg.norm(state)) - 1.0)
        mv0 = self.hamiltonian.matvec_count
        if times[0] == 0.0:
            values[0], bounds[0], serr[0] = observable(state), 0.0, 0.0
            if stored is not None:
                stored[0] = state
            cursor = 1
        t_end = float(times[-1])
        step = min(self.initial_step_us, t_end) if t_end else 0.0
        prefer_max = False
        while cursor < n_t:
            trial = min(step, t_end - now)
            if trial < self.minimum_step_us:
                raise RuntimeError("Lanczos step fell below the configured minimum.")
            snorm = float(np.linalg.norm(state))
            target = self.maximum_dimension if prefer_max else self.minimum_dimension
            v, a, b = self._basis(state, target)
            budget = self.state_error_budget * trial / max(t_end, trial)
            chosen, coef, err = None, None, math.inf
            exact = a.size < target
            if exact:
                chosen, coef, err = a.size, projected_coefficients(a, b, trial), 0.0
            elif not prefer_max:
                coef, err = self._candidate(a, b, self.minimum_dimension, trial, snorm)
                if err <= budget:
                    chosen = self.minimum_dimension
                elif self.maximum_dimension > self.minimum_dimension:
                    v, a, b = self._basis(state, self.maximum_dimension)
                    prefer_max = True
                    exact = a.size < self.maximum_dimension
                    if exact:
                        chosen, coef, err = a.size, projected_coefficients(a, b, trial), 0.0
                    else:
                        for d in self._ladder(self.minimum_dimension + self.dimension_increment):
                            coef, err = self._candidate(a, b, d, trial, snorm)
                            if err <= budget:
                                chosen = d
                                break
            else:
                for d in self._ladder(self.minimum_dimension):
                    coef, err = self._candidate(a, b, d, trial, snorm)
                    if err <= budget:
                        chosen = d
                        break
            if chosen is None or err > budget:
                rejected += 1
                step = 0.5 * trial
                continue
            max_dim = max(max_dim, chosen)
            if chosen > self.minimum_dimension:
                prefer_max = True
            basis = v[:, :chosen]
            gram = observable.project_basis(basis) if projected_ok else None
            hi = _Spectral(a[:chosen], b[: max(0, chosen - 1)])
            low_d = max(1, chosen - self.embedded_offset)
            lo = None if (exact or low_d == chosen) else _Spectral(a[:low_d], b[: max(0, low_d - 1)])
            t_step_end = now + trial
            while cursor < n_t and times[cursor] <= t_step_end + 1e-13:
                dt = float(times[cursor] - now)
                c = hi.coefficients(dt)
                if lo is None:
                    perr = 0.0
                else:
                    diff = c.copy()
                    diff[:low_d] -= lo.coefficients(dt)
                    perr = self.safety_factor * snorm * float(np.linalg.norm(diff))
                if gram is not None:
                    values[cursor] = observable.evaluate_projected(gram, c, snorm)
                    point = None
                else:
                    point = snorm * (basis @ c)
                    values[cursor] = observable(point)
                serr[cursor] = acc_err + perr
                bounds[cursor] = state_error_to_population_bound(serr[cursor])
                if stored is not None:
                    stored[cursor] = point
                cursor += 1
            state = snorm * (basis @ coef)
            now = t_step_end
            acc_err += err
            accepted += 1
            used.append(trial)
            max_norm_err = max(max_norm_err, abs(float(np.linalg.norm(state)) - 1.0))
            if progress_callback is not None:
                progress_callback(now, accepted, rejected, self.hamiltonian.matvec_count - mv0, acc_err)
            step = min(self.maximum_step_us, 1.5 * trial) if err < 0.1 * budget else trial
        stats = PropagationStats(accepted, rejected, self.hamiltonian.matvec_count - mv0, max_dim,
                                 min(used) if used else 0.0, max(used) if used else 0.0, acc_err, max_norm_err)
        return PropagationResult(times, values, bounds, serr, stored, state, stats)


# ---------------------------------------------------------------------------
# Yield quadrature (JD:418-431)
# ---------------------------------------------------------------------------

def simpson(y, x) -> float:
    """Composite Simpson for possibly non-uniform x, as ``scipy.integrate.simpson``.

    Odd point counts use paired parabolic panels; even counts use panels on
    all but the last interval plus the three-point end correction (Cartwright).
    """
    y = np.asarray(y, dtype=float)
    x = np.asarray(x, dtype=float)
    n = y.size
    if n == 1:
        return 0.0
    if n == 2:
        return float(0.5 * (x[1] - x[0]) * (y[0] + y[1]))

    def panels(stop):
        h = np.diff(x)
        h0, h1 = h[0:stop:2], h[1:stop + 1:2]
        hs, hp = h0 + h1, h0 * h1
        r = h0 / h1
        return float(np.sum(hs / 6.0 * (y[0:stop:2] * (2.0 - 1.0 / r) + y[1:stop + 1:2] * (hs * hs / hp)
                                         + y[2:stop + 2:2] * (2.0 - r))))

    if n % 2 == 1:
        return panels(n - 2)
    total = panels(n - 3)
    a, b = x[-2] - x[-3], x[-1] - x[-2]
    alpha = (2 * b * b + 3 * a * b) / (6 * (a + b))
    beta = (b * b + 3 * a * b) / (6 * a)
    eta = b ** 3 / (6 * a * (a + b))
    return total + float(alpha * y[-1] + beta * y[-2] - eta * y[-3])


def integrate_yield(times_us, populations, lifetime_us) -> float:
    """Phi = simpson(exp(-t/tau) P_S / tau, t) (JD:418-420)."""
    t = np.asarray(times_us, dtype=float)
    return simpson(np.exp(-t / lifetime_us) * np.asarray(populations, dtype=float) / lifetime_us, t)


def time_grid_us(maximum_time_us: float, step_us: float = 0.00125) -> np.ndarray:
    """Uniform grid with the endpoint appended when it is not on the grid (JD:325-334)."""
    count = int(math.floor(maximum_time_us / step_us))
    grid = np.arange(count + 1, dtype=float) * step_us
    if grid[-1] < maximum_time_us - 1e-13:
        grid = np.append(grid, maximum_time_us)
    return grid


def coarse_grid_indices(n_points: int, stride: int = 2) -> np.ndarray:
    """Every ``stride``-th point plus the last (JD:423-431)."""
    idx = np.arange(0, n_points, stride, dtype=int)
    if idx[-1] != n_points - 1:
        idx = np.append(idx, n_points - 1)
    return idx


# ---------------------------------------------------------------------------
# Segment propagation (rpm_nuclear_spin_rotation_control.py:281-308)
# ---------------------------------------------------------------------------

def local_unitary_apply(state, dimensions, axis, unitary) -> np.ndarray:
    """d x d operator on one tensor axis (poster_reproduction/core.py:285-292)."""
    t = np.asarray(state, dtype=complex).reshape(tuple(dimensions))
    front = np.moveaxis(t, int(axis), 0)
    out = (np.asarray(unitary, dtype=complex) @ front.reshape(dimensions[axis], -1)).reshape(front.shape)
    return np.moveaxis(out, 0, axis).reshape(-1)


def propagate_segments(initial_state, times_us, segments, *, state_error_budget=2.4e-5, **knobs):
    """The reference's pulsed loop; ``segments`` are (end_us, hamiltonian, pulse|None).

    Returns (values, bounds, final_state, (accepted, rejected, matvecs), accumulated_error).
    """
    times = np.asarray(times_us, dtype=float)
    dims = segments[0][1].dimensions
    obs = SingletPopulationObservable(dims)
    state = np.asarray(initial_state, dtype=complex).reshape(-1)
    values, bounds = np.empty(times.size), np.empty(times.size)
    values[0], bounds[0] = singlet_population(state, dims), 0.0
    cursor, current, acc = 1, 0.0, 0.0
    counts = [0, 0, 0]
    for end, ham, pulse in segments:
        boundary = float(end)
        stop = int(np.searchsorted(times, boundary + 1e-12, side="right"))
        requested = times[cursor:stop] - current
        duration = boundary - current
        local = requested if requested.size and requested[-1] >= duration - 1e-12 else np.append(requested, duration)
        if duration > 0.0:
            prop = AdaptiveLanczosPropagator(ham, **knobs)
            prop.state_error_budget = state_error_budget * duration / times[-1]
            res = prop.propagate(state, local, obs)
            k = requested.size
            values[cursor:stop] = res.observable_values[:k]
            glob = acc + res.state_error_estimates[:k]
            bounds[cursor:stop] = 2.0 * glob + glob ** 2
            state = res.final_state
            counts[0] += res.stats.accepted_steps
            counts[1] += res.stats.rejected_steps
            counts[2] += res.stats.matvecs
            acc += res.stats.accumulated_state_error
        cursor, current = stop, boundary
        if pulse is not None and boundary < times[-1] - 1e-12:
            state = local_unitary_apply(state, dims, pulse[0], pulse[1])
    return values, bounds, state, tuple(counts), acc


# ---------------------------------------------------------------------------
# Entanglement observables of stored states (CORE:311-365)
# ---------------------------------------------------------------------------
def schmidt_values(state, dimensions: Sequence[int], left_axes: Sequence[int]) -> np.ndarray:
    """Singular values of the state reshaped left axes x rest (CORE:317-323)."""
    dims = tuple(int(v) for v in dimensions)
    left = tuple(int(v) for v in left_axes)
    right = tuple(a for a in range(len(dims)) if a not in left)
    tensor = np.asarray(state, dtype=complex).reshape(dims)
    matrix = np.transpose(tensor, left + right).reshape(math.prod(dims[a] for a in left), -1)
    return np.linalg.svd(matrix, compute_uv=False)


def pure_log_negativity(state, dimensions: Sequence[int], left_axes: Sequence[int]) -> float:
    """2 log2 of the sum of normalised Schmidt values (CORE:311-328)."""
    dims = tuple(int(v) for v in dimensions)
    left = tuple(int(v) for v in left_axes)
    if len(set(left)) != len(left) or any(a < 0 or a >= len(dims) for a in left):
        raise ValueError("Invalid subsystem axes.")
    sv = schmidt_values(state, dims, left)
    norm = float(np.linalg.norm(sv))
    if norm == 0.0:
        raise ValueError("Cannot evaluate entanglement of the zero state.")
    return float(2.0 * np.log2(np.sum(sv / norm)))


def reduced_electron_density(state, dimensions: Sequence[int]) -> np.ndarray:
    """Hermitised electron-pair density matrix, state reshaped 4 x rest (CORE:331-334)."""
    m = np.asarray(state, dtype=complex).reshape(4, -1)
    rho = m @ m.conj().T
    return 0.5 * (rho + rho.conj().T)


def mixed_two_electron_log_negativity(rho) -> float:
    """max(0, log2 sum |eig(rho^T_A)|) of a hermitised 4 x 4 matrix (CORE:337-351)."""
    h = 0.5 * (np.asarray(rho, dtype=complex) + np.asarray(rho, dtype=complex).conj().T)
    pt = h.reshape(2, 2, 2, 2).transpose(2, 1, 0, 3).reshape(4, 4)
    return float(max(0.0, np.log2(np.sum(np.abs(np.linalg.eigvalsh(pt))))))


# ---------------------------------------------------------------------------
# Closed-form yields from a dense spectrum
# ---------------------------------------------------------------------------
def _singlet_rows(vectors: np.ndarray, nuclear_dimension: int) -> np.ndarray:
    """Singlet amplitudes (psi[1, k] - psi[2, k]) / sqrt(2) of each column of
    ``vectors`` (electron-major layout, electrons on axes 0 and 1)."""
    m = nuclear_dimension
    return (vectors[m:2 * m] - vectors[2 * m:3 * m]) / math.sqrt(2.0)


def truncated_singlet_yield_dense(h_dense, dimensions: Sequence[int], psi0, lifetime_us: float,
                                  final_time_us: float) -> float:
    """(1/tau) int_0^T exp(-t/tau) P_S(t) dt in closed form for a Hermitian dense H.

    With psi(t) = sum_n c_n exp(-i E_n t)|n> and s_kn the singlet amplitudes of
    eigenvector n, P_S(t) = sum_nm conj(c_n) c_m (s^H s)_nm exp(i (E_n - E_m) t),
    and each term integrates to r (1 - exp(-(r - i w) T)) / (r - i w) with
    r = 1/tau, w = E_n - E_m.  CORE:455-473 (dense_truncated_singlet_yield)
    is the four-level case with the singlet as initial state.
    """
    dims = tuple(int(v) for v in dimensions)
    m = math.prod(dims) // 4
    energies, vectors = np.linalg.eigh(np.asarray(h_dense, dtype=complex))
    coeff = vectors.conj().T @ np.asarray(psi0, dtype=complex)
    rows = _singlet_rows(vectors, m)
    gram = rows.conj().T @ rows
    weights = np.conj(coeff)[:, None] * coeff[None, :] * gram
    rate = 1.0 / float(lifetime_us)
    decay = rate - 1j * (energies[:, None] - energies[None, :])
    integral = rate * (1.0 - np.exp(-decay * float(final_time_us))) / decay
    return float(np.sum(weights * integral).real)


def ensemble_singlet_yield_lorentzian(h_dense, dimensions: Sequence[int], lifetime_us: float) -> float:
    """Infinite-horizon singlet yield of the singlet (x) maximally mixed nuclear
    ensemble from the spectrum: W_nm = |<n|P_S|m>|^2 / M (M nuclear states) and
    sum_nm W_nm / (1 + tau^2 (E_n - E_m)^2) --
    rpm_three_nitrogen_quadrupole.py:100-113 (QuadrupoleModel.spectrum, .yields).
    """
    dims = tuple(int(v) for v in dimensions)
    m = math.prod(dims) // 4
    energies, vectors = np.linalg.eigh(np.asarray(h_dense, dtype=complex))
    rows = _singlet_rows(vectors, m)
    weights = np.abs(rows.conj().T @ rows) ** 2 / m
    gaps2 = (energies[:, None] - energies[None, :]) ** 2
    tau = float(lifetime_us)
    return float(np.sum(weights / (1.0 + tau * tau * gaps2)))


# ---------------------------------------------------------------------------
# Unequal Haberkorn rates (no reference implementation: dense restatement)
# ---------------------------------------------------------------------------
def haberkorn_dense(h_dense, dimensions: Sequence[int], psi0, times_us, singlet_rate: float, triplet_rate: float):
    """Singlet populations and yield under H - (i/2)(kS P_S + kT P_T), dense.

    The state is propagated exactly (eigen-decomposition of the non-Hermitian
    dense operator).  Returns (populations of the state with the common decay
    exp(-min(kS, kT) t / 2) factored out, singlet yield kS int P_S(t) dt on the
    grid by Simpson's rule).  Electrons are axes 0, 1 (C order, slowest).
    """
    dims = tuple(int(v) for v in dimensions)
    n = math.prod(dims)
    m = n // 4
    ps4 = np.zeros((4, 4), dtype=complex)
    ps4[1, 1] = ps4[2, 2] = 0.5
    ps4[1, 2] = ps4[2, 1] = -0.5
    ps = np.kron(ps4, np.eye(m))
    heff = np.asarray(h_dense, dtype=complex) - 0.5j * (singlet_rate * ps + triplet_rate * (np.eye(n) - ps))
    w, v = np.linalg.eig(heff)
    coeff = np.linalg.solve(v, np.asarray(psi0, dtype=complex))
    times = np.asarray(times_us, dtype=float)
    pops = np.empty(times.size)
    for k, t in enumerate(times):
        psi = v @ (np.exp(-1j * w * t) * coeff)
        pops[k] = singlet_population(psi, dims)
    kmin = min(singlet_rate, triplet_rate)
    factored = pops * np.exp(kmin * times)
    yield_value = singlet_rate * simpson(pops, times)
    return factored, yield_value


# ---------------------------------------------------------------------------
# Square field pulse and yield gradients (no reference implementation: dense
# restatement of the segment loop of rpm_nuclear_spin_rotation_control.py:
# 281-308 with per-segment Hamiltonians, and central differences through it)
# ---------------------------------------------------------------------------
def pulsed_yield_dense(h_static, h_pulse, dimensions: Sequence[int], psi0, times_us, pulse_start_us: float,
                       pulse_end_us: float, lifetime_us: float):
    """Singlet populations on a uniform grid and the Simpson yield (JD:418-420)
    for a piecewise-constant Hamiltonian: ``h_pulse`` on observation intervals
    inside [pulse_start, pulse_end], ``h_static`` elsewhere (dense expm of each
    interval propagator; pulse edges on grid points)."""
    from scipy.linalg import expm

    dims = tuple(int(v) for v in dimensions)
    t = np.asarray(times_us, dtype=float)
    dt = float(t[1] - t[0])
    props = (expm(-1j * np.asarray(h_static, dtype=complex) * dt), expm(-1j * np.asarray(h_pulse, dtype=complex) * dt))
    psi = np.asarray(psi0, dtype=complex).copy()
    pops = np.empty(t.size)
    pops[0] = singlet_population(psi, dims)
    for k in range(t.size - 1):
        mid = 0.5 * (t[k] + t[k + 1])
        psi = props[1 if pulse_start_us < mid < pulse_end_us else 0] @ psi
        pops[k + 1] = singlet_population(psi, dims)
    return pops, integrate_yield(t, pops, lifetime_us)


def central_difference(function, params, relative_step: float = 1e-4, richardson: bool = False) -> np.ndarray:
    """Central differences of a scalar function, step relative_step * max(|p|, 1);
    with ``richardson`` the steps h and h/2 are combined, (4 D(h/2) - D(h)) / 3,
    which cancels the O(h^2) truncation term."""
    p = np.asarray(params, dtype=float)
    out = np.empty(p.size)
    for i in range(p.size):
        h = relative_step * max(abs(p[i]), 1.0)

        def diff(step):
            up, down = p.copy(), p.copy()
            up[i] += step
            down[i] -= step
            return (function(up) - function(down)) / (2.0 * step)

        out[i] = (4.0 * diff(0.5 * h) - diff(h)) / 3.0 if richardson else diff(h)
    return out
