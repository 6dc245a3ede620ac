"""Physical constants, spin algebra and local operator builders (host side).

These build the small Hermitian local operators that the device kernels apply.
All frequencies are angular, in rad/us.  Reference behaviour followed (paths
relative to ``Realistic system size/code/`` of sam-not-smart/RPM):

* spin matrices in the descending-m basis: ``rpm_quantum_needle_model.py:178-192``
* zx-plane field vector: ``rpm_quantum_needle_model.py:195-199``
* S.A.I coupling: ``rpm_statevector_engine.py:269-287``
* quadrupole I.Q.I: ``rpm_statevector_engine.py:332-349``
* Efimova-Hore electron pair term: ``rpm_statevector_engine.py:290-329``
* nuclear hyperfine tables: ``rpm_quantum_needle_model.py:37-66``
* nominal quadrupole tensors: ``rpm_quantum_needle_model.py:69-131``
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

TWOPI = 2.0 * math.pi
GAMMA_E_MHZ_PER_MT = 28.0
DEFAULT_FIELD_MICROT = 50.0


def spin_operators(spin: float) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Return (Sx, Sy, Sz) for spin ``spin`` with basis order m = I, ..., -I."""
    d = int(round(2.0 * spin + 1.0))
    m = np.array([spin - k for k in range(d)], dtype=float)
    raise_op = np.zeros((d, d), dtype=complex)
    for col in range(1, d):
        raise_op[col - 1, col] = math.sqrt(spin * (spin + 1.0) - m[col] * (m[col] + 1.0))
    lower_op = raise_op.conj().T
    sx = 0.5 * (raise_op + lower_op)
    sy = -0.5j * (raise_op - lower_op)
    return sx, sy, np.diag(m).astype(complex)


def field_vector_mT(theta_deg: float, field_microT: float = DEFAULT_FIELD_MICROT) -> np.ndarray:
    """Field of ``field_microT`` uT at polar angle theta in the zx plane, in mT."""
    th = math.radians(theta_deg)
    return 1e-3 * field_microT * np.array([math.sin(th), 0.0, math.cos(th)])


def field_vector_spherical_mT(theta_rad: float, phi_rad: float, field_microT: float) -> np.ndarray:
    """Field of ``field_microT`` uT along (theta, phi), in mT (any direction)."""
    st = math.sin(theta_rad)
    return 1e-3 * field_microT * np.array([st * math.cos(phi_rad), st * math.sin(phi_rad), math.cos(theta_rad)])


def zeeman_operator(field_mT: np.ndarray) -> np.ndarray:
    """2 pi gamma_e B.S on one electron (gamma_e = 28 MHz/mT)."""
    s = spin_operators(0.5)
    return TWOPI * GAMMA_E_MHZ_PER_MT * sum(float(b) * op for b, op in zip(field_mT, s))


def two_spin_coupling_operator(left_spin: float, right_spin: float, tensor) -> np.ndarray:
    """Return sum_ab tensor[a, b] S_a (x) I_b."""
    t = np.asarray(tensor, dtype=float)
    if t.shape != (3, 3):
        raise ValueError("A two-spin coupling tensor must be 3x3.")
    left, right = spin_operators(left_spin), spin_operators(right_spin)
    op = np.zeros((left[0].shape[0] * right[0].shape[0],) * 2, dtype=complex)
    for a in range(3):
        for b in range(3):
            if t[a, b] != 0.0:
                op += t[a, b] * np.kron(left[a], right[b])
    return op


def quadrupole_operator(spin: float, tensor) -> np.ndarray:
    """Return the Hermitian single-spin operator sum_ab Q_ab {I_a, I_b}/2."""
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


def efimova_hore_electron_coupling_operator(exchange_J_MHz: float, dipolar_D_MHz: float, dipolar_axis) -> np.ndarray:
    """Electron-pair operator -J (S^2 - 1) + D ((S.n)^2 - S^2/3), in MHz.

    Efimova and Hore, Biophys. J. 94, 1565 (2008), Eqs. 9-10, with the
    state-independent exchange shift kept.
    """
    n = np.asarray(dipolar_axis, dtype=float)
    if n.shape != (3,):
        raise ValueError("dipolar_axis must be a length-3 vector.")
    norm = float(np.linalg.norm(n))
    if norm == 0.0:
        raise ValueError("dipolar_axis must be nonzero.")
    n = n / norm
    one = spin_operators(0.5)
    e2 = np.eye(2, dtype=complex)
    total = [np.kron(op, e2) + np.kron(e2, op) for op in one]
    s_sq = total[0] @ total[0] + total[1] @ total[1] + total[2] @ total[2]
    s_n = n[0] * total[0] + n[1] * total[1] + n[2] * total[2]
    h = -float(exchange_J_MHz) * (s_sq - np.eye(4)) + float(dipolar_D_MHz) * (s_n @ s_n - s_sq / 3.0)
    return 0.5 * (h + h.conj().T)


@dataclass(frozen=True)
class Nucleus:
    """One magnetic nucleus: name, spin and hyperfine tensor in mT."""

    name: str
    spin: float
    tensor_mT: np.ndarray = field(compare=False)

    @property
    def dimension(self) -> int:
        return int(round(2.0 * self.spin + 1.0))


def _t(rows) -> np.ndarray:
    return np.array(rows, dtype=float)


# Hyperfine tensors of the FAD and TrpH radicals (Hiscock et al. SI Tables S1-S2), mT.
FAD_NUCLEI = (
    Nucleus("N5", 1.0, _t([[-0.0989, 0.0039, 0.0], [0.0039, -0.0881, 0.0], [0.0, 0.0, 1.7569]])),
    Nucleus("N10", 1.0, _t([[-0.0190, -0.0048, 0.0], [-0.0048, -0.0196, 0.0], [0.0, 0.0, 0.6046]])),
    Nucleus("H6", 0.5, _t([[-0.2569, -0.1273, 0.0], [-0.1273, -0.4711, 0.0], [0.0, 0.0, -0.4336]])),
    Nucleus("H8a", 0.5, 0.4399 * np.eye(3)),
    Nucleus("H8b", 0.5, 0.4399 * np.eye(3)),
    Nucleus("H8c", 0.5, 0.4399 * np.eye(3)),
    Nucleus("Hbeta", 0.5, 0.4070 * np.eye(3)),
)
TRP_NUCLEI = (
    Nucleus("N1", 1.0, _t([[-0.0336, 0.0924, -0.1354], [0.0924, 0.3303, -0.5318], [-0.1354, -0.5318, 0.6680]])),
    Nucleus("H1", 0.5, _t([[-0.9920, -0.2091, -0.2003], [-0.2091, -0.2631, 0.2803], [-0.2003, 0.2803, -0.5398]])),
    Nucleus("H2", 0.5, _t([[-0.2843, 0.1757, 0.1525], [0.1757, -0.2798, 0.0975], [0.1525, 0.0975, -0.2699]])),
    Nucleus("H4", 0.5, _t([[-0.5596, -0.1956, -0.1657], [-0.1956, -0.4020, 0.0762], [-0.1657, 0.0762, -0.5021]])),
    Nucleus("H5", 0.5, _t([[0.0051, 0.0616, 0.0694], [0.0616, -0.0665, 0.0391], [0.0694, 0.0391, -0.0586]])),
    Nucleus("H7", 0.5, _t([[-0.4355, -0.1541, -0.1239], [-0.1541, -0.2777, 0.0864], [-0.1239, 0.0864, -0.3770]])),
    Nucleus("Hbeta1", 0.5, _t([[1.5808, -0.0453, -0.0506], [-0.0453, 1.5575, 0.0988], [-0.0506, 0.0988, 1.6752]])),
)
ALL_NUCLEI = FAD_NUCLEI + TRP_NUCLEI
NUCLEAR_RADICALS = ("FAD",) * len(FAD_NUCLEI) + ("TrpH",) * len(TRP_NUCLEI)
SPIN_ORDER = ("eA", "eB") + tuple(f"{r}:{n.name}" for r, n in zip(NUCLEAR_RADICALS, ALL_NUCLEI))
SYSTEM_DIMENSIONS = (2, 2) + tuple(n.dimension for n in ALL_NUCLEI)
NUCLEAR_DIMENSION = math.prod(SYSTEM_DIMENSIONS[2:])
STATE_DIMENSION = math.prod(SYSTEM_DIMENSIONS)


def _q_on_hyperfine_axes(hf: np.ndarray, principal, orientation: str) -> np.ndarray:
    """Traceless quadrupole tensor whose principal axes are the hyperfine axes.

    ``ring_normal`` puts Qzz on the hyperfine axis of largest |A|;
    ``ring_plane_provisional`` puts it on the first in-plane axis and Qyy on
    the normal.
    """
    p = np.asarray(principal, dtype=float)
    p = p - p.mean()
    evals, evecs = np.linalg.eigh(hf)
    normal = int(np.argmax(np.abs(evals)))
    plane = [k for k in range(3) if k != normal]
    values = np.empty(3)
    if orientation == "ring_normal":
        values[normal], values[plane[0]], values[plane[1]] = p[2], p[0], p[1]
    elif orientation == "ring_plane_provisional":
        values[plane[0]], values[plane[1]], values[normal] = p[2], p[0], p[1]
    else:
        raise ValueError(f"Unknown quadrupole orientation: {orientation}")
    q = evecs @ np.diag(values) @ evecs.T
    return 0.5 * (q + q.T)


# Efimova & Hore, Mol. Phys. 107, 665 (2009), Table 2: principal values in mT.
QUADRUPOLE_PRINCIPAL_VALUES_MT = {
    "FAD:N5": (0.031, 0.041, -0.072),
    "FAD:N10": (0.032, 0.041, -0.072),
    "TrpH:N1": (0.016, 0.020, -0.036),
}
QUADRUPOLE_TENSORS_MT = {
    "FAD:N5": _q_on_hyperfine_axes(FAD_NUCLEI[0].tensor_mT, QUADRUPOLE_PRINCIPAL_VALUES_MT["FAD:N5"], "ring_plane_provisional"),
    "FAD:N10": _q_on_hyperfine_axes(FAD_NUCLEI[1].tensor_mT, QUADRUPOLE_PRINCIPAL_VALUES_MT["FAD:N10"], "ring_normal"),
    "TrpH:N1": _q_on_hyperfine_axes(TRP_NUCLEI[0].tensor_mT, QUADRUPOLE_PRINCIPAL_VALUES_MT["TrpH:N1"], "ring_normal"),
}
