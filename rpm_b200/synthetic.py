"""Seeded synthetic radical-pair systems and workloads.

The benchmark workloads are self-contained: hyperfine and quadrupole tensors,
electron couplings, field orientations and random-phase initial vectors are
all drawn from NumPy's PCG64 generator with recorded seeds.  The same term
list feeds the GPU engine and the CPU oracle.

Distributions:

* hyperfine ``A = a 1 + T``: ``a ~ U(-1, 1)`` mT, ``T`` symmetric traceless
  built from entries ``~ N(0, 0.3)`` mT (symmetrised, trace removed);
* spin-1 quadrupole: principal values ``(e2qQ/h)/4 * (-(1-eta), -(1+eta), 2)``
  with ``e2qQ/h ~ U(0.5, 3)`` MHz and ``eta ~ U(0, 0.5)``, rotated by a random
  SO(3) rotation and converted to rad/us (x 2 pi);
* electron pair: Efimova-Hore form with ``D`` and ``J`` given in mT and
  converted at gamma_e = 28 MHz/mT (the reference's constant stands for
  g = 2.0023), dipolar axis a random unit vector;
* nuclei are ordered spin-1 first within each radical, FAD before TrpH, so the
  full system has the reference dimensions (2,2,3,3,2,2,2,2,2,3,2,2,2,2,2,2).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .model import (
    GAMMA_E_MHZ_PER_MT,
    TWOPI,
    efimova_hore_electron_coupling_operator,
    field_vector_spherical_mT,
    quadrupole_operator,
    two_spin_coupling_operator,
    zeeman_operator,
)


@dataclass(frozen=True)
class SyntheticNucleus:
    radical: str  # "FAD" or "TrpH"
    spin: float
    hyperfine_mT: np.ndarray = field(compare=False)
    quadrupole_rad_per_us: np.ndarray | None = field(default=None, compare=False)

    @property
    def dimension(self) -> int:
        return int(round(2 * self.spin + 1))


def random_rotation(rng: np.random.Generator) -> np.ndarray:
    """Uniform random SO(3) matrix (QR of a Gaussian matrix with sign fix)."""
    q, r = np.linalg.qr(rng.normal(size=(3, 3)))
    q = q * np.sign(np.diag(r))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def draw_hyperfine(rng: np.random.Generator) -> np.ndarray:
    iso = rng.uniform(-1.0, 1.0)
    t = rng.normal(0.0, 0.3, size=(3, 3))
    t = 0.5 * (t + t.T)
    t -= np.trace(t) / 3.0 * np.eye(3)
    return iso * np.eye(3) + t


def draw_quadrupole(rng: np.random.Generator) -> np.ndarray:
    cq = rng.uniform(0.5, 3.0)
    eta = rng.uniform(0.0, 0.5)
    principal = 0.25 * cq * np.array([-(1.0 - eta), -(1.0 + eta), 2.0])
    rot = random_rotation(rng)
    q = rot @ np.diag(principal) @ rot.T
    return TWOPI * 0.5 * (q + q.T)


def random_unit_vector(rng: np.random.Generator) -> np.ndarray:
    v = rng.normal(size=3)
    return v / np.linalg.norm(v)


@dataclass
class SyntheticSystem:
    """A seeded radical pair; call :meth:`terms` for a field orientation."""

    seed: int
    nuclei: tuple
    exchange_J_mT: float
    dipolar_D_mT: float
    dipolar_axis: np.ndarray
    field_microT: float = 50.0

    @property
    def dimensions(self) -> tuple[int, ...]:
        return (2, 2) + tuple(n.dimension for n in self.nuclei)

    @property
    def dimension(self) -> int:
        return math.prod(self.dimensions)

    @property
    def left_axes(self) -> tuple[int, ...]:
        return (0,) + tuple(k + 2 for k, n in enumerate(self.nuclei) if n.radical == "FAD")

    @property
    def right_axes(self) -> tuple[int, ...]:
        return (1,) + tuple(k + 2 for k, n in enumerate(self.nuclei) if n.radical == "TrpH")

    def terms(self, theta_rad: float, phi_rad: float = 0.0, *, field_microT: float | None = None,
              hyperfine_scale: float = 1.0, extra_field_mT=None):
        """Local terms (axes, operator, label) in rad/us for one field direction."""
        from .engine import LocalTerm

        b = field_vector_spherical_mT(theta_rad, phi_rad, self.field_microT if field_microT is None else field_microT)
        if extra_field_mT is not None:
            b = b + np.asarray(extra_field_mT, dtype=float)
        z = zeeman_operator(b)
        out = [LocalTerm((0,), z, "electron A Zeeman"), LocalTerm((1,), z, "electron B Zeeman")]
        for k, n in enumerate(self.nuclei):
            e = 0 if n.radical == "FAD" else 1
            hf = TWOPI * GAMMA_E_MHZ_PER_MT * hyperfine_scale * two_spin_coupling_operator(0.5, n.spin, n.hyperfine_mT)
            out.append(LocalTerm((e, k + 2), hf, f"{n.radical}:{k} hyperfine"))
            if n.quadrupole_rad_per_us is not None:
                out.append(LocalTerm((k + 2,), quadrupole_operator(n.spin, n.quadrupole_rad_per_us), f"{n.radical}:{k} quadrupole"))
        pair = TWOPI * efimova_hore_electron_coupling_operator(
            self.exchange_J_mT * GAMMA_E_MHZ_PER_MT, self.dipolar_D_mT * GAMMA_E_MHZ_PER_MT, self.dipolar_axis)
        if np.any(pair != 0.0):
            out.append(LocalTerm((0, 1), pair, "electron exchange + dipolar"))
        return out


def make_system(seed: int, fad: tuple[int, int], trp: tuple[int, int], *, exchange_J_mT=None,
                dipolar_D_mT: float = -0.4, field_microT: float = 50.0) -> SyntheticSystem:
    """Draw a system with ``fad = (n_spin1, n_spin_half)`` and ``trp`` likewise.

    ``exchange_J_mT=None`` draws ``J ~ U(-0.1, 0.1)`` mT.
    """
    rng = np.random.default_rng(int(seed))
    nuclei = []
    for radical, (n1, nh) in (("FAD", fad), ("TrpH", trp)):
        for _ in range(n1):
            hf = draw_hyperfine(rng)
            nuclei.append(SyntheticNucleus(radical, 1.0, hf, draw_quadrupole(rng)))
        for _ in range(nh):
            nuclei.append(SyntheticNucleus(radical, 0.5, draw_hyperfine(rng)))
    j = rng.uniform(-0.1, 0.1) if exchange_J_mT is None else float(exchange_J_mT)
    axis = random_unit_vector(rng)
    return SyntheticSystem(int(seed), tuple(nuclei), j, float(dipolar_D_mT), axis, field_microT)


def prefix_system(full: SyntheticSystem, per_radical: int) -> SyntheticSystem:
    """Equal-count nuclear prefixes of both radicals (as the reference selects baths)."""
    fad = [n for n in full.nuclei if n.radical == "FAD"][:per_radical]
    trp = [n for n in full.nuclei if n.radical == "TrpH"][:per_radical]
    return SyntheticSystem(full.seed, tuple(fad + trp), full.exchange_J_mT, full.dipolar_D_mT,
                           full.dipolar_axis, full.field_microT)


def fibonacci_sphere(n: int) -> list[tuple[float, float]]:
    """``n`` quasi-uniform (theta, phi) directions."""
    golden = math.pi * (3.0 - math.sqrt(5.0))
    return [(math.acos(1.0 - 2.0 * (k + 0.5) / n), (k * golden) % (2 * math.pi)) for k in range(n)]


# Workload presets ---------------------------------------------------------

SMALL_SEED = 96
FULL_SEED = 221184


def small_system() -> SyntheticSystem:
    """2 electrons + 1 spin-1 + 3 spin-1/2 nuclei: dimension 96, J = 0, D = -0.4 mT."""
    return make_system(SMALL_SEED, (1, 1), (0, 2), exchange_J_mT=0.0)


def full_system() -> SyntheticSystem:
    """2 electrons + 11 spin-1/2 + 3 spin-1 nuclei: dimension 221,184."""
    return make_system(FULL_SEED, (2, 5), (1, 6))


def random_phase_vectors(dimensions, count: int, seed: int) -> np.ndarray:
    """``count`` singlet (x) random-phase vectors, shape (count, N), complex128."""
    dims = tuple(dimensions)
    m = math.prod(dims[2:])
    rng = np.random.default_rng(int(seed))
    out = np.zeros((count, 4 * m), dtype=complex)
    s = 1.0 / math.sqrt(2.0)
    for k in range(count):
        nuc = np.exp(1j * rng.uniform(0.0, TWOPI, m)) / math.sqrt(m)
        out[k, m:2 * m] = s * nuc
        out[k, 2 * m:3 * m] = -s * nuc
    return out
