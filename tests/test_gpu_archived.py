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
    # A budget 100x tighter than the archived runs'.  Over this 57.56-us
    # horizon (about ten times the 5-us benchmark horizon) the complex64
    # H psi has an accuracy floor of about 1e-6 in the yield: the FP32
    # rounding of the Hamiltonian's coefficients is a fixed relative
    # perturbation of H (~6e-8) whose phase error grows with time.  A
    # tight-budget FP64 run of the last row agrees with its archived yield to
    # 3e-12, so the archived yields are the reference and the bar is their
    # own estimate plus that floor.
    FP32_FLOOR = 1.5e-6
    bp = BatchedPropagator(hams, krylov_dimension=32, state_error_budget=2.4e-7)
    out = bp.propagate([init] * len(ROWS), times, system_index=list(range(len(ROWS))), lifetime_us=TAU)
    errs = []
    for r, y in zip(ROWS, out.yields):
        tol = float(r["yield_propagation_estimate"]) + float(r["quadrature_error"]) + FP32_FLOOR
        errs.append(abs(y - float(r["yield"])))
        assert errs[-1] < tol, (r, y)
    assert float(np.sqrt(np.mean(np.square(errs)))) < 1e-6
