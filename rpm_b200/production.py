"""Production assembly, seeds and the yield integral (drop-in host API).

Mirrors (paths relative to ``Realistic system size/code/``):

* ``build_quantum_needle_hamiltonian`` -- rpm_statevector_engine.py:367-469
* ``build_hamiltonian`` / ``make_propagator`` / ``random_phase_initial_state``
  -- poster_reproduction/core.py:172-258
* ``_seed`` / ``integrate_yield`` / ``coarse_grid_indices`` / ``SweepConfig``
  time grid -- rpm_quantum_needle_jd_sweeps.py:307-431
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _lib
from .engine import (
    AdaptiveLanczosPropagator,
    CompiledFullPairHamiltonian,
    LocalTerm,
    MatrixFreeHamiltonian,
    _torch,
)
from .model import (
    ALL_NUCLEI,
    FAD_NUCLEI,
    GAMMA_E_MHZ_PER_MT,
    NUCLEAR_RADICALS,
    QUADRUPOLE_TENSORS_MT,
    SPIN_ORDER,
    SYSTEM_DIMENSIONS,
    TWOPI,
    Nucleus,
    efimova_hore_electron_coupling_operator,
    field_vector_mT,
    quadrupole_operator,
    spin_operators,
    two_spin_coupling_operator,
)

MASTER_SEED = 20260731
R2_D_PAPER_UT = -2783.0 / 8.0  # Efimova-Hore D in equivalent-field uT


def equivalent_field_uT_to_MHz(value_uT: float) -> float:
    return float(value_uT) * GAMMA_E_MHZ_PER_MT / 1000.0


@dataclass(frozen=True)
class ElectronCoupling:
    """Efimova-Hore D and J in equivalent-field uT with the dipolar axis."""

    d_paper_uT: float = 0.0
    exchange_J_uT: float = 0.0
    dipolar_axis: tuple[float, float, float] = (1.0, 0.0, 0.0)

    @classmethod
    def ratio(cls, d_over_j: float) -> "ElectronCoupling":
        if float(d_over_j) == 0.0:
            raise ValueError("Efimova-Hore D/J ratio cannot be zero.")
        return cls(R2_D_PAPER_UT, R2_D_PAPER_UT / float(d_over_j))

    @property
    def d_paper_MHz(self) -> float:
        return equivalent_field_uT_to_MHz(self.d_paper_uT)

    @property
    def exchange_J_MHz(self) -> float:
        return equivalent_field_uT_to_MHz(self.exchange_J_uT)


UNCOUPLED = ElectronCoupling()
PRODUCTION_COUPLING = ElectronCoupling.ratio(-3.0)


def _zeeman(theta_deg: float, field_microT: float) -> np.ndarray:
    s = spin_operators(0.5)
    b = field_vector_mT(theta_deg, field_microT)
    return TWOPI * GAMMA_E_MHZ_PER_MT * (b[0] * s[0] + b[1] * s[1] + b[2] * s[2])


def build_quantum_needle_hamiltonian(theta_deg: float, field_microT: float = 50.0, *, exchange_J_MHz: float = 0.0,
                                     dipolar_tensor_MHz: np.ndarray | None = None,
                                     efimova_hore_D_MHz: float | None = None,
                                     efimova_hore_axis: np.ndarray | None = None,
                                     quadrupole_scale: float = 1.0) -> MatrixFreeHamiltonian:
    """Full radical-pair Hamiltonian with optional electron couplings (ENG:367-469)."""
    zeeman = _zeeman(theta_deg, field_microT)
    terms = [LocalTerm((0,), zeeman, "electron A Zeeman"), LocalTerm((1,), zeeman, "electron B Zeeman")]
    for k, nucleus in enumerate(ALL_NUCLEI):
        e = 0 if k < len(FAD_NUCLEI) else 1
        hf = TWOPI * GAMMA_E_MHZ_PER_MT * two_spin_coupling_operator(0.5, nucleus.spin, nucleus.tensor_mT)
        terms.append(LocalTerm((e, k + 2), hf, f"{nucleus.name} hyperfine"))
        q = QUADRUPOLE_TENSORS_MT.get(SPIN_ORDER[k + 2])
        if q is not None and quadrupole_scale != 0.0:
            terms.append(LocalTerm((k + 2,), quadrupole_operator(
                nucleus.spin, TWOPI * GAMMA_E_MHZ_PER_MT * float(quadrupole_scale) * q), f"{nucleus.name} nuclear quadrupole"))
    if efimova_hore_D_MHz is not None and dipolar_tensor_MHz is not None:
        raise ValueError("Choose either dipolar_tensor_MHz or efimova_hore_D_MHz, not both.")
    if efimova_hore_D_MHz is not None:
        axis = np.array([1.0, 0.0, 0.0]) if efimova_hore_axis is None else np.asarray(efimova_hore_axis, dtype=float)
        op = TWOPI * efimova_hore_electron_coupling_operator(exchange_J_MHz, efimova_hore_D_MHz, axis)
        if np.any(op != 0.0):
            terms.append(LocalTerm((0, 1), op, "Efimova-Hore electron exchange + dipolar coupling"))
        return MatrixFreeHamiltonian(SYSTEM_DIMENSIONS, terms)
    dipolar = np.zeros((3, 3)) if dipolar_tensor_MHz is None else np.asarray(dipolar_tensor_MHz, dtype=float)
    if dipolar.shape != (3, 3):
        raise ValueError("dipolar_tensor_MHz must be a 3x3 tensor.")
    tensor = TWOPI * (dipolar - 2.0 * float(exchange_J_MHz) * np.eye(3))
    if np.any(tensor != 0.0):
        terms.append(LocalTerm((0, 1), two_spin_coupling_operator(0.5, 0.5, tensor), "electron exchange + dipolar coupling"))
    return MatrixFreeHamiltonian(SYSTEM_DIMENSIONS, terms)


def dimensions_for(nuclei: Sequence[Nucleus]) -> tuple[int, ...]:
    return (2, 2) + tuple(n.dimension for n in nuclei)


ENTANGLEMENT_NUCLEAR_COUNTS = (4, 6, 8, 10, 12, 14)


def selected_nuclei(nuclear_count: int) -> tuple[Nucleus, ...]:
    """Equal strongest-first prefixes of the two radicals (core.py:135-142)."""
    if int(nuclear_count) not in ENTANGLEMENT_NUCLEAR_COUNTS:
        raise ValueError(f"nuclear_count must be one of {ENTANGLEMENT_NUCLEAR_COUNTS}.")
    per = int(nuclear_count) // 2
    return tuple(FAD_NUCLEI[:per] + ALL_NUCLEI[len(FAD_NUCLEI):][:per])


def selected_radicals(nuclear_count: int) -> tuple[str, ...]:
    per = int(nuclear_count) // 2
    return ("FAD",) * per + ("TrpH",) * per


@dataclass(frozen=True)
class _BathSite:
    """One nucleus of the bath: its tensor axis, the electron of its radical
    (0 = FAD / electron A, 1 = TrpH / electron B) and its "radical:name" key."""

    axis: int
    electron: int | None
    key: str
    nucleus: Nucleus


_RADICAL_ELECTRON = {"FAD": 0, "TrpH": 1}


def _bath_sites(nuclei: Sequence[Nucleus], radicals: Sequence[str]) -> list[_BathSite]:
    """Validated site table of a bath prefix.  Error texts and their order are
    the ones callers of core.py:172-229 match on: a length mismatch first,
    then duplicate keys, then a radical other than FAD / TrpH."""
    if len(nuclei) != len(radicals):
        raise ValueError("nuclei and radicals must have the same length.")
    sites = [_BathSite(axis, _RADICAL_ELECTRON.get(radical), f"{radical}:{nucleus.name}", nucleus)
             for axis, (nucleus, radical) in enumerate(zip(nuclei, radicals), start=2)]
    keys = [site.key for site in sites]
    if len(set(keys)) != len(keys):
        raise ValueError("Selected nuclei contain duplicate radical/name keys.")
    if any(site.electron is None for site in sites):
        raise ValueError("Every selected nucleus must belong to FAD or TrpH.")
    return sites


def production_terms(theta_deg: float, field_mT: float, *, coupling: ElectronCoupling = PRODUCTION_COUPLING,
                     quadrupole_scale: float = 1.0, nuclei: Sequence[Nucleus] = ALL_NUCLEI,
                     radicals: Sequence[str] = NUCLEAR_RADICALS,
                     hyperfine_overrides_mT: dict[str, np.ndarray] | None = None):
    """(dimensions, terms, left_axes, right_axes) of the production
    Hamiltonian; host-only, see :func:`build_hamiltonian`.

    Same operator and term labels as core.py:172-229 (labels and error texts
    are matched by callers); assembled from the validated site table: the two
    electron Zeeman terms, then per site its hyperfine term and, where the
    site has a quadrupole tensor and the scale is nonzero, its quadrupole
    term, then the electron-pair coupling.  The radical split groups each
    electron with the sites of its radical.
    """
    sites = _bath_sites(nuclei, radicals)
    overrides = hyperfine_overrides_mT or {}
    to_rad = TWOPI * GAMMA_E_MHZ_PER_MT  # mT -> rad/us
    zeeman = _zeeman(theta_deg, float(field_mT) * 1000.0)
    terms = [LocalTerm((e,), zeeman, f"electron {name} Zeeman") for e, name in ((0, "A"), (1, "B"))]
    for site in sites:
        hf_tensor = np.asarray(overrides.get(site.key, site.nucleus.tensor_mT), dtype=float)
        terms.append(LocalTerm((site.electron, site.axis),
                               to_rad * two_spin_coupling_operator(0.5, site.nucleus.spin, hf_tensor),
                               f"{site.key} hyperfine"))
        q_tensor = QUADRUPOLE_TENSORS_MT.get(site.key)
        if q_tensor is not None and quadrupole_scale != 0.0:
            terms.append(LocalTerm((site.axis,), quadrupole_operator(site.nucleus.spin, to_rad * quadrupole_scale * q_tensor),
                                   f"{site.key} quadrupole"))
    pair = efimova_hore_electron_coupling_operator(coupling.exchange_J_MHz, coupling.d_paper_MHz,
                                                   np.asarray(coupling.dipolar_axis, dtype=float))
    terms.append(LocalTerm((0, 1), TWOPI * pair, "Efimova-Hore exchange + full nonsecular dipolar"))
    split = {e: (e,) + tuple(site.axis for site in sites if site.electron == e) for e in (0, 1)}
    return dimensions_for(nuclei), terms, split[0], split[1]


def build_hamiltonian(theta_deg: float, field_mT: float, *, coupling: ElectronCoupling = PRODUCTION_COUPLING,
                      quadrupole_scale: float = 1.0, nuclei: Sequence[Nucleus] = ALL_NUCLEI,
                      radicals: Sequence[str] = NUCLEAR_RADICALS,
                      hyperfine_overrides_mT: dict[str, np.ndarray] | None = None) -> CompiledFullPairHamiltonian:
    """Production non-factorised Hamiltonian of any paired bath prefix on the
    device (core.py:172-229; term list from :func:`production_terms`)."""
    dims, terms, left, right = production_terms(theta_deg, field_mT, coupling=coupling,
                                                quadrupole_scale=quadrupole_scale, nuclei=nuclei, radicals=radicals,
                                                hyperfine_overrides_mT=hyperfine_overrides_mT)
    return CompiledFullPairHamiltonian(dims, terms, left_axes=left, right_axes=right)


def make_propagator(hamiltonian, *, state_error_budget: float = 2.4e-5, minimum_dimension: int = 24,
                    maximum_dimension: int = 64, dimension_increment: int = 8, embedded_offset: int = 4,
                    safety_factor: float = 2.0, initial_step_us: float = 0.05,
                    maximum_step_us: float = 0.25) -> AdaptiveLanczosPropagator:
    """Production Krylov settings (core.py:232-247 with the SweepConfig defaults)."""
    return AdaptiveLanczosPropagator(hamiltonian, minimum_dimension=minimum_dimension,
                                     maximum_dimension=maximum_dimension, dimension_increment=dimension_increment,
                                     embedded_offset=embedded_offset, safety_factor=safety_factor,
                                     state_error_budget=state_error_budget, initial_step_us=initial_step_us,
                                     maximum_step_us=maximum_step_us)


def _seed(base: int, sample_id: int) -> int:
    """First uint32 of SeedSequence([base, 0xA11CE, sample]) (jd_sweeps.py:373-375)."""
    return int(np.random.SeedSequence([int(base), 0xA11CE, int(sample_id)]).generate_state(1, dtype=np.uint32)[0])


sample_seed = _seed


def random_phase_initial_state(dimensions: Sequence[int], master_seed: int, sample_id: int) -> np.ndarray:
    """Singlet (x) seeded random-phase nuclear state (core.py:250-258)."""
    rng = np.random.default_rng(_seed(master_seed, sample_id))
    m = math.prod(dimensions[2:])
    nuclei = np.exp(1.0j * rng.uniform(0.0, TWOPI, m)) / math.sqrt(m)
    out = np.zeros(4 * m, dtype=complex)
    out[m:2 * m] = nuclei / math.sqrt(2.0)
    out[2 * m:3 * m] = -nuclei / math.sqrt(2.0)
    return out


def full_product_basis_indices(master_seed: int, sample_id: int) -> tuple[int, ...]:
    """One reproducible computational product state of the 14 nuclei (core.py:261-265)."""
    rng = np.random.default_rng(sample_seed(master_seed, sample_id))
    return tuple(int(rng.integers(d)) for d in SYSTEM_DIMENSIONS[2:])


def paired_product_indices(nuclear_count: int, full_indices: Sequence[int]) -> tuple[int, ...]:
    """The FAD and TrpH prefixes of a 14-nucleus product state (core.py:280-282)."""
    per = int(nuclear_count) // 2
    return tuple(full_indices[:per]) + tuple(full_indices[7:7 + per])


def product_basis_initial_state(dimensions: Sequence[int], indices: Sequence[int]) -> np.ndarray:
    """Electron singlet x one nuclear computational basis state (core.py:268-277)."""
    dims = tuple(int(v) for v in dimensions)
    if len(indices) != len(dims) - 2:
        raise ValueError("One product-basis index is required per nuclear axis.")
    nuclei = np.zeros(math.prod(dims[2:]), dtype=complex)
    nuclei[int(np.ravel_multi_index(tuple(int(i) for i in indices), dims[2:]))] = 1.0
    singlet = np.array([0.0, 1.0, -1.0, 0.0], dtype=complex) / math.sqrt(2.0)
    return np.kron(singlet, nuclei)


def entanglement_time_grids_us() -> tuple[np.ndarray, np.ndarray]:
    """Nested fine/coarse grids of the 0-2 us entanglement average (core.py:107-126).

    Fine: 0-0.1 us every 0.000125 us, then every 0.0025 us to 2 us; coarse:
    twice both spacings, an exact subset (its indices into the fine grid are
    returned).
    """
    fine = np.concatenate((np.arange(0.0, 0.1 + 0.0000625, 0.000125), np.arange(0.1025, 2.0 + 0.00125, 0.0025)))
    coarse = np.concatenate((np.arange(0.0, 0.1 + 0.000125, 0.00025), np.arange(0.105, 2.0 + 0.0025, 0.005)))
    fine[-1] = coarse[-1] = 2.0
    indices = np.searchsorted(fine, coarse)
    if not np.allclose(fine[indices], coarse, rtol=0.0, atol=1e-13):
        raise RuntimeError("Entanglement quadrature grids are not nested.")
    return fine, indices


def integrate_yield(times_us, populations, lifetime_us: float) -> float:
    """Phi = simpson(exp(-t/tau) P_S(t) / tau, t) in FP64 on the GPU (jd_sweeps.py:418-420)."""
    torch = _torch()
    t = torch.as_tensor(np.asarray(times_us, dtype=float), device="cuda")
    p = torch.as_tensor(np.asarray(populations, dtype=float), device="cuda")
    if t.ndim != 1 or p.shape != t.shape:
        raise ValueError("If given, length of x along axis must be the same as y.")
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    _lib.call("rpm_simpson_yield", _lib.ptr(t), _lib.ptr(p), int(t.numel()), 1, int(t.numel()), float(lifetime_us),
              _lib.ptr(out), _lib.stream_handle())
    return float(out.item())


def time_grid_us(maximum_time_us: float, integration_step_us: float = 0.00125) -> np.ndarray:
    """Uniform grid to T with the endpoint appended when off-grid (jd_sweeps.py:325-334)."""
    count = int(math.floor(maximum_time_us / integration_step_us))
    grid = np.arange(count + 1, dtype=float) * integration_step_us
    if grid[-1] < maximum_time_us - 1e-13:
        grid = np.append(grid, maximum_time_us)
    return grid


def maximum_time_us(lifetime_us: float, survival_tail_bound: float) -> float:
    """T = -tau ln(tail) (jd_sweeps.py:325-327)."""
    return -lifetime_us * math.log(survival_tail_bound)


def coarse_grid_indices(n_points: int, integration_step_us: float = 0.00125,
                        coarse_integration_step_us: float = 0.0025) -> np.ndarray:
    """Nested coarse-grid indices (jd_sweeps.py:423-431)."""
    ratio = coarse_integration_step_us / integration_step_us
    stride = int(round(ratio))
    if stride < 1 or not math.isclose(ratio, stride, rel_tol=0.0, abs_tol=1e-12):
        raise ValueError("The coarse integration step must be an integer fine-grid multiple.")
    idx = np.arange(0, n_points, stride, dtype=int)
    if idx[-1] != n_points - 1:
        idx = np.append(idx, n_points - 1)
    return idx
