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
