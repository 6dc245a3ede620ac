"""Validation record of the CPU baseline's prefix extrapolation.

CPU-baseline measurement infrastructure, not product code.  The benchmark's
CPU baseline times short prefixes of the 5-us horizon and extrapolates
linearly.  This script records, once, on the host it runs on:

* the oracle port (the code ``bench.py`` times on the GPU box) and, when the
  reference checkout is given, the reference's own
  ``CompiledFullPairHamiltonian`` + ``AdaptiveLanczosPropagator`` +
  ``SingletPopulationObservable`` (rpm_statevector_engine.py:132-266,
  500-538, 612-933), imported unchanged;
* each on a 0.25-us prefix (state-error budget scaled by 0.25/5, as
  rpm_full14_quadrupole_experiment.py:138-148 scales it) and on the full
  5-us trajectory, at the plain path's budget 1e-10 and at the batched
  path's budget 5e-7;

with the benchmark's workload: the 221,184-dimensional synthetic FAD-TrpH
system at theta = pi/4, phi = 0, one random-phase vector, Krylov dimensions
8-40.  It writes ``oracle/cpu_extrapolation.json``: wall seconds, matvecs,
the prefix extrapolated to 5 us and its ratio to the full run, and the
port / reference time ratio.  Every case runs in its own spawned process
with one BLAS thread.

    python oracle/cpu_extrapolation.py [<RPM checkout>]
"""

from __future__ import annotations

import json
import math
import multiprocessing as mp
import os
import platform
import sys
import time
import types
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent
HORIZON_US = 5.0
PREFIX_US = 0.25
GRID_US = 0.00125
SEED = 77


def _stub_matplotlib():
    mpl = types.ModuleType("matplotlib")
    mpl.use = lambda *a, **k: None
    pyplot = types.ModuleType("matplotlib.pyplot")
    pyplot.__getattr__ = lambda name: (lambda *a, **k: None)
    mpl.pyplot = pyplot
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", pyplot)


def _run(case):
    impl, horizon, budget, reference = case
    for var in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[var] = "1"
    sys.path.insert(0, str(REPO))
    import numpy as np

    from rpm_b200 import synthetic

    if impl == "reference":
        sys.path.insert(0, str(Path(reference) / "Realistic system size" / "code"))
        _stub_matplotlib()
        import rpm_statevector_engine as eng  # noqa: N813
    else:
        import oracle as eng
    full = synthetic.full_system()
    terms = [eng.LocalTerm(t.axes, np.asarray(t.operator, dtype=complex), t.label)
             for t in full.terms(math.pi / 4, 0.0)]
    h = eng.CompiledFullPairHamiltonian(full.dimensions, terms, left_axes=full.left_axes,
                                        right_axes=full.right_axes)
    psi = synthetic.random_phase_vectors(full.dimensions, 1, SEED)[0]
    times = np.arange(int(round(horizon / GRID_US)) + 1) * GRID_US
    prop = eng.AdaptiveLanczosPropagator(h, minimum_dimension=8, maximum_dimension=40, dimension_increment=8,
                                         embedded_offset=4, state_error_budget=budget * horizon / HORIZON_US)
    t0 = time.perf_counter()
    res = prop.propagate(psi, times, eng.SingletPopulationObservable(full.dimensions))
    wall = time.perf_counter() - t0
    return {"impl": impl, "horizon_us": horizon, "budget": budget, "seconds": wall,
            "matvecs": int(res.stats.matvecs), "accepted_steps": int(res.stats.accepted_steps)}


def main(reference: str | None) -> None:
    impls = ["port"] + (["reference"] if reference else [])
    cases = [(impl, hz, budget, reference) for impl in impls for budget in (1e-10, 5e-7)
             for hz in (PREFIX_US, HORIZON_US)]
    with mp.get_context("spawn").Pool(min(len(cases), os.cpu_count() or 1)) as pool:
        rows = pool.map(_run, cases)
    summary = []
    for impl in impls:
        for budget in (1e-10, 5e-7):
            pre = next(r for r in rows if r["impl"] == impl and r["budget"] == budget and r["horizon_us"] == PREFIX_US)
            ful = next(r for r in rows if r["impl"] == impl and r["budget"] == budget and r["horizon_us"] == HORIZON_US)
            extrap = pre["seconds"] * HORIZON_US / PREFIX_US
            summary.append({"impl": impl, "budget": budget, "prefix_s": pre["seconds"], "full_s": ful["seconds"],
                            "prefix_extrapolated_s": extrap, "full_over_extrapolated": ful["seconds"] / extrap,
                            "prefix_matvecs": pre["matvecs"], "full_matvecs": ful["matvecs"]})
    ratios = {}
    if reference:
        for budget in (1e-10, 5e-7):
            p = next(s for s in summary if s["impl"] == "port" and s["budget"] == budget)
            r = next(s for s in summary if s["impl"] == "reference" and s["budget"] == budget)
            ratios[str(budget)] = {"port_over_reference_prefix": p["prefix_s"] / r["prefix_s"],
                                   "port_over_reference_full": p["full_s"] / r["full_s"]}
    out = {"workload": "221,184-dim synthetic FAD-TrpH system, theta = pi/4, phi = 0, one random-phase vector "
                       f"(seed {SEED}), Krylov 8-40 (increment 8, offset 4), 0.00125-us grid",
           "host": {"cpu": platform.processor() or platform.machine(), "cores": os.cpu_count(),
                    "python": platform.python_version()},
           "prefix_us": PREFIX_US, "horizon_us": HORIZON_US, "runs": rows, "summary": summary,
           "port_over_reference": ratios}
    (HERE / "cpu_extrapolation.json").write_text(json.dumps(out, indent=1) + "\n")
    print(json.dumps(summary, indent=1))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else None)
