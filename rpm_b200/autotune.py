"""Autotuner of the batched propagator: Krylov dimension, trajectory tile,
reorthogonalisation policy and step budget.

The batched path (:class:`rpm_b200.batched.BatchedPropagator`) has knobs whose
best values depend on the systems and the GPU:

* the Krylov dimension m (cost per Krylov step grows about linearly in m,
  the step the embedded error estimate allows grows faster than m);
* the trajectory tile, i.e. how many trajectories one batch carries (larger
  tiles amortise the per-step controller and fill the GPU; the Krylov basis
  costs ``tile * (m + 1) * ld * 8`` bytes);
* the reorthogonalisation policy of the complex64 Lanczos recurrence: none
  (Paige's three-term form) or periodic (every P iterations the next vector
  is reorthogonalised against the whole basis, two classical Gram-Schmidt
  passes; the reference reorthogonalises every iteration,
  rpm_statevector_engine.py:675-676);
* the state-error budget.  The reference's bound on the population error is
  ``2 eps + eps**2`` (rpm_statevector_engine.py:541-543), and a yield is a
  weighted average of populations with weights of total at most one, so a
  yield tolerance ``tol`` admits ``eps <= tol / 2``; the tuner never picks a
  looser budget.

Each candidate runs the real batched propagation for a prefix of the
horizon with the budget scaled by prefix / horizon, so that every Krylov step
meets the same local tolerance as in the full run (the Hamiltonian is time
independent, so the cost per simulated microsecond is stationary), and is
scored in trajectory-microseconds per second.  A candidate is eligible only if
its prefix yields agree with a tight-budget run of the same trajectories
within ``accuracy`` (half the yield tolerance by default): speed never buys
accuracy.  Trial trajectories are drawn round-robin over the
sample's shapes (system dimensions), so uneven batches are represented.
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
REORTH_POLICIES = (0, 16)            # reorthogonalisation period (0: none)


@dataclass
class TuneResult:
    krylov_dimension: int
    tile: int
    state_error_budget: float
    throughput: float                 # trajectory-us simulated per second at the chosen point
    reorth_period: int = 0
    trials: list = field(default_factory=list)

    def propagator(self, hamiltonians, **kwargs) -> BatchedPropagator:
        """A BatchedPropagator configured with the tuned knobs."""
        return BatchedPropagator(hamiltonians, krylov_dimension=self.krylov_dimension,
                                 state_error_budget=self.state_error_budget, reorth_period=self.reorth_period,
                                 **kwargs)

    def to_json(self) -> str:
        return json.dumps(asdict(self))


def budget_for_yield_tolerance(tolerance: float) -> float:
    """Largest accumulated state-error budget whose population bound meets ``tolerance``."""
    if not tolerance > 0.0:
        raise ValueError("yield tolerance must be positive")
    return 0.5 * tolerance


def spread_selection(system_index: Sequence[int], shape_of: Sequence, count: int) -> np.ndarray:
    """``count`` sample positions drawn round-robin over the shapes of the
    sample (in order of first appearance), each shape's positions in order."""
    idx = np.asarray(system_index)
    groups: dict = {}
    for pos, k in enumerate(idx):
        groups.setdefault(shape_of[int(k)], []).append(pos)
    queues = [list(v) for v in groups.values()]
    out = []
    while len(out) < min(count, idx.size):
        for q in queues:
            if q and len(out) < count:
                out.append(q.pop(0))
    return np.asarray(sorted(out), dtype=np.int64)


def _run(hams, states, system_index, times, m, budget, reorth, repeats, lifetime, kernel):
    """(best seconds, prefix yields) of one candidate."""
    torch = _torch()
    bp = BatchedPropagator(hams, krylov_dimension=m, state_error_budget=budget, reorth_period=reorth,
                           lanczos_kernel=kernel)
    order = bp.shape_order(system_index)
    idx = np.asarray(system_index) if order is None else np.asarray(system_index)[order]
    sts = states if order is None else [states[k] for k in order]
    psi0 = bp.load_states(sts, idx)
    work = torch.empty_like(psi0)
    work.copy_(psi0)
    bp.propagate_device(work, times, idx)  # warm-up: graph capture, buffers
    best, values = float("inf"), None
    for _ in range(repeats):
        work.copy_(psi0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        values, _, stats = bp.propagate_device(work, times, idx)
        torch.cuda.synchronize()
        best = min(best, time.perf_counter() - t0)
        if any(s.status for s in stats):
            return best, None
    yields = bp.yields_device(times, values, lifetime).cpu().numpy()
    if order is not None:
        inverse = np.empty_like(order)
        inverse[order] = np.arange(order.size)
        yields = yields[inverse]
    return best, yields


def tune(hamiltonians: Sequence, states, system_index: Sequence[int], *, horizon_us: float = 0.25,
         full_horizon_us: float = 5.0, grid_us: float = 0.00125, yield_tolerance: float = 1e-6,
         accuracy: float | None = None, krylov_dimensions: Sequence[int] = KRYLOV_RANGE,
         tiles: Sequence[int] | None = None, reorth_periods: Sequence[int] = (0,), repeats: int = 1,
         memory_fraction: float = 0.6, lifetime_us: float = 1.0, lanczos_kernel: str = "persistent",
         cache: str | Path | None = None) -> TuneResult:
    """Pick (Krylov dimension, tile, reorthogonalisation period, budget) for
    trajectories ``states`` of ``hamiltonians``.

    ``states``/``system_index`` are a representative sample of the workload
    (at least as many trajectories as the largest tile tried).  Each
    candidate propagates ``tile`` of them, spread over the sample's shapes,
    over ``horizon_us`` with the budget scaled to that prefix; it is eligible
    when its prefix yields are within ``accuracy`` (default: half the yield
    tolerance) of a run at a hundredth of the budget with the largest Krylov
    dimension.  Tiles whose Krylov basis would need more
    than ``memory_fraction`` of the free device memory are skipped.  With
    ``cache`` the result is stored in (and reused from) that JSON file, keyed
    by the systems' dimensions, the device name and the search space.
    """
    torch = _torch()
    hams = list(hamiltonians)
    idx = np.asarray(system_index, dtype=np.int32)
    if idx.size == 0:
        raise ValueError("at least one sample trajectory is required")
    budget = budget_for_yield_tolerance(yield_tolerance)
    accuracy = 0.5 * yield_tolerance if accuracy is None else float(accuracy)
    tiles = tuple(sorted({t for t in (tiles or TILE_RANGE) if t <= idx.size} or {int(idx.size)}))
    reorths = tuple(int(p) for p in reorth_periods)
    key = json.dumps({"dims": sorted({h.dimension for h in hams}), "device": torch.cuda.get_device_name(),
                      "m": list(krylov_dimensions), "tiles": list(tiles), "reorth": list(reorths), "budget": budget,
                      "horizon": horizon_us, "full": full_horizon_us, "accuracy": accuracy})
    if cache is not None:
        path = Path(cache)
        if path.exists():
            stored = json.loads(path.read_text())
            if key in stored:
                return TuneResult(**stored[key])
    times = np.arange(int(round(horizon_us / grid_us)) + 1) * grid_us
    frac = horizon_us / full_horizon_us
    trial_budget = budget * frac
    gate = accuracy
    ld = max(h.dimension for h in hams)
    shapes = [(tuple(h.dimensions), tuple(getattr(h, "left_axes", ()))) for h in hams]
    # tight-budget reference yields of every trajectory any tile uses
    pool = spread_selection(idx, shapes, max(tiles))
    _, ref_y = _run(hams, [states[k] for k in pool], idx[pool], times, max(krylov_dimensions), trial_budget / 100.0,
                    0, 1, lifetime_us, lanczos_kernel)
    ref_of = {int(p): y for p, y in zip(pool, ref_y)}
    free, _ = torch.cuda.mem_get_info()
    trials = []
    best = None
    for m in krylov_dimensions:
        for reorth in reorths:
            for tile in tiles:
                trial = {"krylov_dimension": m, "tile": tile, "reorth_period": reorth}
                need = tile * (m + 1) * ld * 8 + tile * ld * 32
                if need > memory_fraction * free:
                    trials.append({**trial, "skipped": "memory"})
                    continue
                sel = pool[spread_selection(idx[pool], shapes, tile)]
                secs, ys = _run(hams, [states[k] for k in sel], idx[sel], times, m, trial_budget, reorth, repeats,
                                lifetime_us, lanczos_kernel)
                rate = tile * horizon_us / secs
                err = float(np.max(np.abs(ys - np.array([ref_of[int(p)] for p in sel])))) if ys is not None else None
                ok = err is not None and err <= gate
                trials.append({**trial, "seconds": secs, "throughput": rate, "yield_err_prefix": err, "accepted": ok})
                if ok and (best is None or rate > best[0]):
                    best = (rate, m, tile, reorth)
    if best is None:
        raise RuntimeError("no autotuner candidate fits in device memory and meets the accuracy gate")
    result = TuneResult(krylov_dimension=best[1], tile=best[2], state_error_budget=budget, throughput=best[0],
                        reorth_period=best[3], trials=trials)
    if cache is not None:
        path = Path(cache)
        stored = json.loads(path.read_text()) if path.exists() else {}
        stored[key] = asdict(result)
        path.write_text(json.dumps(stored, indent=1))
    return result


@dataclass
class ShapeTuning:
    """Per-shape tuning of an uneven batch: each shape group's Krylov
    dimension (the batch's per-system caps) and tile."""
    shapes: list                      # shape key of each group, in order of first appearance
    results: list                     # TuneResult of each group
    caps: list                        # Krylov dimension of each Hamiltonian (its group's)
    state_error_budget: float

    @property
    def krylov_dimension(self) -> int:
        return max(self.caps)

    def chunks(self, counts: Sequence[int]) -> int:
        """Launches needed when each launch carries at most one tile of every group."""
        return max(-(-int(c) // r.tile) for c, r in zip(counts, self.results))

    def propagator(self, hamiltonians, **kwargs) -> BatchedPropagator:
        reorth = max(r.reorth_period for r in self.results)
        return BatchedPropagator(hamiltonians, krylov_dimension=self.krylov_dimension,
                                 state_error_budget=self.state_error_budget, krylov_caps=self.caps,
                                 reorth_period=reorth, **kwargs)


def tune_per_shape(hamiltonians: Sequence, states, system_index: Sequence[int], *,
                   tiles: Sequence[int] | None = None, **knobs) -> ShapeTuning:
    """:func:`tune` run on each shape group of the sample alone (its own
    trajectories, tiles up to its size), so that an uneven batch gives every
    system size its own Krylov dimension and tile.  ``knobs`` are passed on to
    :func:`tune`."""
    hams = list(hamiltonians)
    idx = np.asarray(system_index, dtype=np.int32)
    shapes = [(tuple(h.dimensions), tuple(getattr(h, "left_axes", ()))) for h in hams]
    order: list = []
    for k in idx:
        if shapes[int(k)] not in order:
            order.append(shapes[int(k)])
    results = []
    for shape in order:
        pos = [p for p, k in enumerate(idx) if shapes[int(k)] == shape]
        group = sorted({int(idx[p]) for p in pos})
        local = {k: i for i, k in enumerate(group)}
        cand = tuple(t for t in (tiles or TILE_RANGE) if t <= len(pos)) or (len(pos),)
        results.append(tune([hams[k] for k in group], [states[p] for p in pos],
                            [local[int(idx[p])] for p in pos], tiles=cand, **knobs))
    caps = [results[order.index(shapes[k])].krylov_dimension if shapes[k] in order else 0 for k in range(len(hams))]
    return ShapeTuning(shapes=[list(map(list, s)) for s in order], results=results, caps=caps,
                       state_error_budget=results[0].state_error_budget)
