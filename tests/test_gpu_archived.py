"""Reproduce the reference's archived full-size production yields on the GPU.

tests/golden/archived_full14_yields.json holds rows of the reference's
results/quadrupole/full14_uncoupled_tau5_29angles/raw_sample_yields.csv
(221,184-dim production Hamiltonian, 50 uT, tau = 5 us, T = 57.56 us, Krylov
24-64, budget 2.4e-5, seed 20260731, sample 0).  Each archived yield carries
its propagation-error estimate (about 1e-6) and quadrature error.
"""

import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROWS = json.loads((Path(__file__).parent / "golden" / "archived_full14_yields.json").read_text())
TAU = 5.0
HORIZON = -TAU * np.log(1e-5)


def _hamiltonian(row):
    import rpm_b200 as rb
    from rpm_b200.production import PRODUCTION_COUPLING, UNCOUPLED

    coupling = UNCOUPLED if row["electron_interactions"] == "D=J=0" else PRODUCTION_COUPLING
    return rb.build_hamiltonian(float(row["theta_deg"]), 0.05, coupling=coupling,
                                quadrupole_scale=float(row["scale"]))


def test_plain_fp64_path_reproduces_an_archived_yield():
    import rpm_b200 as rb
    from rpm_b200.production import time_grid_us

    row = ROWS[0]  # D = J = 0, Q = 0, theta = 0
    h = _hamiltonian(row)
    init = rb.random_phase_initial_state(h.dimensions, 20260731, int(row["sample_id"]))
    times = time_grid_us(HORIZON)
    res = rb.make_propagator(h).propagate(init, times, rb.SingletPopulationObservable(h.dimensions))
    y = rb.integrate_yield(times, res.observable_values, TAU)
    # the plain path repeats the reference's decisions; only ulp-level initial-state
    # differences between NumPy builds separate the two runs
    assert abs(y - float(row["yield"])) < 1e-8


def test_batched_path_reproduces_all_archived_yields():
    import rpm_b200 as rb
    from rpm_b200.batched import BatchedPropagator
    from rpm_b200.production import time_grid_us

    hams = [_hamiltonian(r) for r in ROWS]
    dims = hams[0].dimensions
    init = rb.random_phase_initial_state(dims, 20260731, 0)
    times = time_grid_us(HORIZON)
    # a budget 100x tighter than the archived runs', so that the comparison is
    # limited by the archived yields' own error estimate
    bp = BatchedPropagator(hams, krylov_dimension=32, state_error_budget=2.4e-7)
    out = bp.propagate([init] * len(ROWS), times, system_index=list(range(len(ROWS))), lifetime_us=TAU)
    for r, y in zip(ROWS, out.yields):
        tol = float(r["yield_propagation_estimate"]) + float(r["quadrature_error"]) + 1e-7
        assert abs(y - float(r["yield"])) < tol, (r, y)
