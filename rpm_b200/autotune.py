"""Autotuner of the batched propagator: Krylov dimension, trajectory tile and step budget.

The batched path (:class:`rpm_b200.batched.BatchedPropagator`) has three
knobs whose best values depend on the systems and the GPU:

* the Krylov dimension m (cost per Krylov step grows about linearly in m,
  the step the embedded error estimate allows grows faster than m);
* the trajectory tile, i.e. how many trajectories one batch carries (larger
  tiles amortise the per-step controller, which runs one CTA per trajectory,
  and fill the GPU; the Krylov basis costs ``tile * (m + 1) * ld * 8`` bytes);
* the state-error budget.  The reference's bound on the population error is
  ``2 eps + eps**2`` (rpm_statevector_engine.py:541-543), and a yield is a
  weighted average of populations with weights of total at most one, so a
  yield tolerance ``tol`` admits ``eps <= tol / 2``; the tuner never picks a
  looser budget.

Each candidate runs the real batched propagation for a short prefix of the
horizon (the Hamiltonian is time independent, so the cost per simulated
microsecond is stationary) and is scored in trajectory-microseconds per
second.  The Lanczos recurrence is Paige's three-term form without
reorthogonalisation: the complex64 rounding floor of the basis, not loss of
orthogonality, limits the yields (measured against the FP64 path), so no
reorthogonalisation policy is offered.
"""

from __future__ import annotations

import json
import time
from dataclasses import asdict, dataclass, field
from pathlib import Path
from typing import Sequence

import numpy as np

from .batched import BatchedPropagator
from .engine import _torch

KRYLOV_RANGE = (16, 24, 32, 40)      # the batched configuration's Krylov cap range
# Every cap the batched path accepts (its limit is 64): larger caps take
# longer Krylov steps for the same per-step controller work.
KRYLOV_EXTENDED = (16, 24, 32, 40, 48, 56, 64)
TILE_RANGE = (8, 16, 32, 48, 64)     # trajectories per batch


@dataclass
class TuneResult:
    krylov_dimension: int
    tile: int
    state_error_budget: float
    throughput: float                 # trajectory-us simulated per second at the chosen point
    trials: list = field(default_factory=list)

    def propagator(self, hamiltonians, **kwargs) -> BatchedPropagator:
        """A BatchedPropagator configured with the tuned knobs."""
        return BatchedPropagator(hamiltonians, krylov_dimension=self.krylov_dimension,
                                 state_error_budget=self.state_error_budget, **kwargs)

    def to_json(self) -> str:
        return json.dumps(asdict(self))


def budget_for_yield_tolerance(tolerance: float) -> float:
    """Largest accumulated state-error budget whose population bound meets ``tolerance``."""
    if not tolerance > 0.0:
        raise ValueError("yield tolerance must be positive")
    return 0.5 * tolerance


def _trial(hams, states, system_index, times, m: int, budget: float, repeats: int) -> float:
    torch = _torch()
    bp = BatchedPropagator(hams, krylov_dimension=m, state_error_budget=budget)
    psi0 = bp.load_states(states, system_index)
    work = torch.empty_like(psi0)
    work.copy_(psi0)
    bp.propagate_device(work, times, system_index)  # warm-up: graph capture, buffers
    best = float("inf")
    for _ in range(repeats):
        work.copy_(psi0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        bp.propagate_device(work, times, system_index)
        torch.cuda.synchronize()
        best = min(best, time.perf_counter() - t0)
    return best


def tune(hamiltonians: Sequence, states, system_index: Sequence[int], *, horizon_us: float = 0.25,
         grid_us: float = 0.00125, yield_tolerance: float = 1e-6, krylov_dimensions: Sequence[int] = KRYLOV_RANGE,
         tiles: Sequence[int] | None = None, repeats: int = 1, memory_fraction: float = 0.6,
         cache: str | Path | None = None) -> TuneResult:
    """Pick (Krylov dimension, tile, budget) for trajectories ``states`` of ``hamiltonians``.

    ``states``/``system_index`` are a representative sample of the workload
    (at least as many trajectories as the largest tile tried); the trial
    propagates them over ``horizon_us``.  Tiles whose Krylov basis would need
    more than ``memory_fraction`` of the free device memory are skipped.  With
    ``cache`` the result is stored in (and reused from) that JSON file, keyed
    by the systems' dimensions, the device name and the search space.
    """
    torch = _torch()
    hams = list(hamiltonians)
    idx = np.asarray(system_index, dtype=np.int32)
    if idx.size == 0:
        raise ValueError("at least one sample trajectory is required")
    budget = budget_for_yield_tolerance(yield_tolerance)
    tiles = tuple(sorted({t for t in (tiles or TILE_RANGE) if t <= idx.size} or {int(idx.size)}))
    key = json.dumps({"dims": sorted({h.dimension for h in hams}), "device": torch.cuda.get_device_name(),
                      "m": list(krylov_dimensions), "tiles": list(tiles), "budget": budget, "horizon": horizon_us})
    if cache is not None:
        path = Path(cache)
        if path.exists():
            stored = json.loads(path.read_text())
            if key in stored:
                return TuneResult(**stored[key])
    times = np.arange(int(round(horizon_us / grid_us)) + 1) * grid_us
    ld = max(h.dimension for h in hams)
    free, _ = torch.cuda.mem_get_info()
    trials = []
    best = None
    for m in krylov_dimensions:
        for tile in tiles:
            need = tile * (m + 1) * ld * 8 + tile * ld * 32
            if need > memory_fraction * free:
                trials.append({"krylov_dimension": m, "tile": tile, "skipped": "memory"})
                continue
            sel = np.arange(tile)
            secs = _trial(hams, [states[k] for k in sel], idx[sel], times, m, budget, repeats)
            rate = tile * horizon_us / secs
            trials.append({"krylov_dimension": m, "tile": tile, "seconds": secs, "throughput": rate})
            if best is None or rate > best[0]:
                best = (rate, m, tile)
    if best is None:
        raise RuntimeError("no autotuner candidate fits in device memory")
    result = TuneResult(krylov_dimension=best[1], tile=best[2], state_error_budget=budget, throughput=best[0],
                        trials=trials)
    if cache is not None:
        path = Path(cache)
        stored = json.loads(path.read_text()) if path.exists() else {}
        stored[key] = asdict(result)
        path.write_text(json.dumps(stored, indent=1))
    return result
