"""Trajectory cells in the reference's checkpoint format.

One ``.npz`` cell per trajectory with the keys the reference's full-size
runner writes (``rpm_full14_quadrupole_experiment.py:154-194``): fine and
coarse Simpson yields, quadrature error, the propagation-error estimate
(Simpson of the survival-weighted population bounds), the tail bound, the
populations and their bounds on the time grid, state-error estimates, the
final state, the initial singlet population and ``metadata_json`` (with the
``configuration_hash`` a resume is checked against).  Files are written
atomically (temporary file + ``os.replace``), as the reference does
(F14:131-135), so GPU trajectories feed the existing reports unchanged.
"""

from __future__ import annotations

import hashlib
import json
import math
import os
from pathlib import Path

import numpy as np

CELL_KEYS = ("yield", "coarse_yield", "quadrature_error", "yield_propagation_estimate", "yield_tail_bound",
             "times_us", "singlet_population", "population_error_estimate", "state_error_estimates", "final_state",
             "initial_singlet", "metadata_json")


def configuration_hash(config: dict) -> str:
    """SHA-256 of the configuration serialised with sorted keys (F14 digest style)."""
    return hashlib.sha256(json.dumps(config, sort_keys=True).encode()).hexdigest()


def cell_values(times_us, populations, bounds, state_errors, *, lifetime_us: float, tail_bound: float,
                coarse_stride: int = 2) -> dict:
    """Yield figures of one trajectory, integrated on the GPU (FP64 Simpson)."""
    from .production import integrate_yield

    times = np.asarray(times_us, dtype=float)
    pops = np.asarray(populations, dtype=float)
    idx = np.arange(0, times.size, coarse_stride, dtype=int)
    if idx[-1] != times.size - 1:
        idx = np.append(idx, times.size - 1)
    fine = integrate_yield(times, pops, lifetime_us)
    coarse = integrate_yield(times[idx], pops[idx], lifetime_us)
    estimate = integrate_yield(times, np.asarray(bounds, dtype=float), lifetime_us)
    return {"yield": np.array(fine), "coarse_yield": np.array(coarse), "quadrature_error": np.array(abs(fine - coarse)),
            "yield_propagation_estimate": np.array(estimate), "yield_tail_bound": np.array(tail_bound),
            "times_us": times, "singlet_population": pops,
            "population_error_estimate": np.asarray(bounds, dtype=float),
            "state_error_estimates": np.asarray(state_errors, dtype=float)}


def write_cell(path, values: dict, *, final_state, initial_singlet: float, metadata: dict) -> Path:
    """Write one cell atomically; ``values`` comes from :func:`cell_values`."""
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    payload = dict(values)
    payload["final_state"] = np.asarray(final_state)
    payload["initial_singlet"] = np.array(float(initial_singlet))
    payload["metadata_json"] = np.array(json.dumps(metadata, sort_keys=True))
    missing = [k for k in CELL_KEYS if k not in payload]
    if missing:
        raise ValueError(f"cell is missing {missing}")
    tmp = path.with_suffix(path.suffix + f".{os.getpid()}.tmp")
    with tmp.open("wb") as stream:
        np.savez_compressed(stream, **payload)
    os.replace(tmp, path)
    return path


def read_cell(path, *, expected_hash: str | None = None) -> tuple[dict, dict]:
    """Load a cell; raise ValueError if its configuration hash differs or a yield
    figure is not finite (the reference's resume checks)."""
    with np.load(Path(path), allow_pickle=False) as data:
        values = {k: data[k] for k in data.files}
    metadata = json.loads(str(values["metadata_json"]))
    if expected_hash is not None and metadata.get("configuration_hash") != expected_hash:
        raise ValueError(f"Incompatible checkpoint: {path}")
    for key in ("yield", "quadrature_error", "yield_propagation_estimate", "yield_tail_bound"):
        if not np.isfinite(float(values[key])):
            raise ValueError(f"Nonfinite checkpoint: {path}")
    return values, metadata


# ---------------------------------------------------------------------------
# The full-size runner's configuration and its digest
# ---------------------------------------------------------------------------
F14_ANGLES = (0.0, 80.0, 85.0, 88.0, 89.0, 90.0, 91.0, 92.0, 95.0, 100.0, 180.0)
F14_SCALES = (0.0, 1.0)


def f14_stable_dict(*, seed: int | None = None, samples: int = 4, angles_deg=F14_ANGLES, field_mT: float = 0.05,
                    lifetime_us: float = 5.0, tail_bound: float = 1e-5, integration_step_us: float = 0.00125,
                    coarse_step_us: float = 0.0025, state_error_budget: float = 2.4e-5,
                    bootstrap_replicates: int = 2000, smoke: bool = False) -> dict:
    """The configuration record whose digest the full-size runner stores in
    every cell and checks on resume (rpm_full14_quadrupole_experiment.py:46-92).

    Its keys, values and their JSON form are the reference's file format (a
    resume compares digests), so they are reproduced exactly: the runner's
    configuration fields, the tensor dimensions and axis labels of the bath
    (the smoke bath is FAD N5, N10 and TrpH N1), the quadrupole scales and
    tensors, the hyperfine tensors, the Efimova-Hore D/J = -3 coupling record,
    the horizon -tau ln(tail bound), the production Krylov settings and the
    fixed descriptive strings.
    """
    from .model import ALL_NUCLEI, FAD_NUCLEI, NUCLEAR_RADICALS, QUADRUPOLE_TENSORS_MT
    from .production import MASTER_SEED, R2_D_PAPER_UT, dimensions_for, equivalent_field_uT_to_MHz

    if smoke:
        trp_first = ALL_NUCLEI[len(FAD_NUCLEI)]
        nuclei, radicals = (FAD_NUCLEI[0], FAD_NUCLEI[1], trp_first), ("FAD", "FAD", "TrpH")
    else:
        nuclei, radicals = ALL_NUCLEI, NUCLEAR_RADICALS
    ratio = -3.0
    token = f"{ratio:+.6f}".replace("+", "p").replace("-", "m").replace(".", "p")
    coupling = {"condition_id": f"eh_R_{token}", "family": "efimova_hore", "role": "paper_cancellation_scan",
                "d_paper_uT": R2_D_PAPER_UT, "exchange_J_uT": R2_D_PAPER_UT / ratio, "ratio_D_over_J": ratio,
                "dipolar_axis": [1.0, 0.0, 0.0], "convention": "Efimova-Hore Eqs. 9-10",
                "d_paper_MHz": equivalent_field_uT_to_MHz(R2_D_PAPER_UT),
                "exchange_J_MHz": equivalent_field_uT_to_MHz(R2_D_PAPER_UT / ratio)}
    fields = {"seed": MASTER_SEED if seed is None else int(seed), "samples": samples,
              "angles_deg": list(angles_deg), "field_mT": field_mT, "lifetime_us": lifetime_us,
              "tail_bound": tail_bound, "integration_step_us": integration_step_us, "coarse_step_us": coarse_step_us,
              "state_error_budget": state_error_budget, "bootstrap_replicates": bootstrap_replicates, "smoke": smoke}
    return {**fields, "schema_version": 1, "dimensions": list(dimensions_for(nuclei)),
            "ordering": ["eA", "eB"] + [f"{r}:{n.name}" for n, r in zip(nuclei, radicals)],
            "full_coupled_pair": True, "factorized_evolution": False,
            "quadrupole_scales": list(F14_SCALES),
            "quadrupole_tensors_mT": {k: np.asarray(v).tolist() for k, v in QUADRUPOLE_TENSORS_MT.items()},
            "quadrupole_orientation": "existing molecular-frame tensors; N5 in-plane azimuth provisional, not fitted",
            "hyperfine_tensors_mT": {f"{r}:{n.name}": np.asarray(n.tensor_mT).tolist()
                                     for n, r in zip(nuclei, radicals)},
            "coupling": coupling,
            "maximum_time_us": -lifetime_us * math.log(tail_bound),
            "krylov": {"min_dimension": 24, "max_dimension": 64, "increment": 8, "embedded_offset": 4,
                       "safety_factor": 2.0, "initial_step_us": 0.05, "max_step_us": 0.25,
                       "state_error_budget": state_error_budget},
            "initial_state": "electronic singlet times seeded nuclear random phase; common seeds across Q and angle",
            "relaxation": False, "nuclear_Zeeman": False}


def f14_digest(**config) -> str:
    """SHA-256 of :func:`f14_stable_dict` in the runner's JSON form (sorted
    keys, default separators), the ``configuration_hash`` of its cells."""
    return configuration_hash(f14_stable_dict(**config))
