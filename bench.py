"""Benchmark: radical-pair trajectories/s at 221,184 dimensions.

Default arm (``--impl b200``): the batched mixed-precision GPU path over the
full-size FAD-TrpH-shaped synthetic radical pair, 12 Fibonacci-sphere field
orientations x V random-phase vectors per step, propagated to 5 us on the
0.00125-us grid with the singlet yield (tau = 1 us).  One "step" is one such
batch.  ``value`` is whole-job trajectories/s with the states resident in HBM;
``e2e`` is the same through the public Python API from pinned host buffers.
Beside it: the plain single-vector FP64 GPU path on one trajectory (the
reference's controller, Krylov 8-40, budget 1e-10) and the yield error of the
batched path against it, the H psi roofline, and the CPU baseline (the
oracle's NumPy/SciPy port of the reference's FP64 path on all host cores, on a
bounded prefix of the horizon).

Reference arm (``--impl reference``): that CPU port alone, on the host cores.

Multi-GPU (torchrun): every rank propagates its own batch (weak scaling, no
data-path collective); per-trajectory yields are all-gathered at the end.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

METRIC = "RP trajectories/s at 221,184-dim, batched vs plain GPU, yield err ≤1e-6"
UNIT = "trajectories/s"
HORIZON_US = 5.0
GRID_US = 0.00125
LIFETIME_US = 1.0
YIELD_TOL = 1e-6  # singlet-yield error bar of the metric
FALLBACK_HBM_GBS = 6650.0
WORKLOAD = ("221,184-dim synthetic FAD-TrpH-shaped radical pair (2 e + 11 spin-1/2 + 3 spin-1), random-phase "
            "trajectories to 5 us on the 0.00125-us grid (4001 points), singlet yield tau = 1 us, yield error <= 1e-6")


# ---------------------------------------------------------------------------
# CPU baseline (oracle port): one spawned process per host core, each owning
# one trajectory that it advances segment by segment
# ---------------------------------------------------------------------------
def _cpu_worker_main(conn, seed: int, budget: float) -> None:
    for var in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[var] = "1"
    import numpy as np

    import oracle
    from rpm_b200 import synthetic

    full = synthetic.full_system()
    terms = full.terms(math.pi / 4, 0.0)
    h = oracle.CompiledFullPairHamiltonian(full.dimensions, [oracle.LocalTerm(t.axes, t.operator) for t in terms],
                                           left_axes=full.left_axes, right_axes=full.right_axes)
    observable = oracle.SingletPopulationObservable(full.dimensions)
    psi = synthetic.random_phase_vectors(full.dimensions, 1, seed)[0]
    conn.send("ready")
    while True:
        duration = conn.recv()
        if duration is None:
            break
        # the state carries over from the previous segment (H is time independent);
        # the budget is scaled by the segment's share of the 5-us horizon
        times = np.arange(int(round(duration / GRID_US)) + 1) * GRID_US
        prop = oracle.AdaptiveLanczosPropagator(h, minimum_dimension=8, maximum_dimension=40,
                                                state_error_budget=budget * duration / HORIZON_US)
        t0 = time.perf_counter()
        res = prop.propagate(psi, times, observable)
        psi = res.final_state
        conn.send((time.perf_counter() - t0, int(res.stats.matvecs)))
    conn.close()


class CpuBaseline:
    """The oracle's FP64 port (the reference's controller, Krylov 8-40) on
    `workers` host processes with one BLAS thread each, every process
    propagating its own trajectory of the benchmark system at theta = pi/4."""

    def __init__(self, workers: int, budget: float, seed0: int = 77):
        import multiprocessing as mp

        ctx = mp.get_context("spawn")
        self.workers, self.budget = workers, budget
        self.conns, self.procs = [], []
        for k in range(workers):
            parent, child = ctx.Pipe()
            proc = ctx.Process(target=_cpu_worker_main, args=(child, seed0 + k, budget), daemon=True)
            proc.start()
            self.conns.append(parent)
            self.procs.append(proc)
        for c in self.conns:
            if c.recv() != "ready":
                raise RuntimeError("CPU baseline worker failed to start")
        self.simulated_us = 0.0
        self.matvecs = 0

    def segment(self, duration_us: float) -> float:
        """Advance every worker's trajectory by `duration_us`; wall seconds."""
        t0 = time.perf_counter()
        for c in self.conns:
            c.send(float(duration_us))
        out = [c.recv() for c in self.conns]
        self.simulated_us += duration_us
        self.matvecs += sum(o[1] for o in out)
        return time.perf_counter() - t0

    def close(self):
        for c in self.conns:
            try:
                c.send(None)
            except OSError:
                pass
        for p in self.procs:
            p.join(timeout=30)


def extrapolation_record():
    """The committed once-only validation of the prefix extrapolation
    (oracle/cpu_extrapolation.json, written by oracle/cpu_extrapolation.py)."""
    path = ROOT / "oracle" / "cpu_extrapolation.json"
    try:
        rec = json.loads(path.read_text())
    except (OSError, ValueError):
        return None
    return {"source": "oracle/cpu_extrapolation.json", "host": rec.get("host"), "summary": rec.get("summary"),
            "port_over_reference": rec.get("port_over_reference")}


def cpu_workers() -> int:
    n = os.cpu_count() or 1
    return max(1, min(n, 64))


# ---------------------------------------------------------------------------
# Clock sampling during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_uuid: str | None):
        self.proc = None
        self.lines: list[str] = []
        try:
            cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
            if device_uuid:
                cmd += ["-i", device_uuid]
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], 0.0, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax = max(smax, float(parts[1]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[3:7]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm():
    path = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(path.read_text())["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError):
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic_per_vector(fused: bool):
    """DRAM bytes per vector of the dominant launch pair (one fused Lanczos
    iteration, or one H psi for the general cube kernels) from the committed
    ncu summary, or None."""
    name = "lanczos_iteration_fused_c64.md" if fused else "hpsi_cube_c64_batched.md"
    path = ROOT / "profiles" / name
    try:
        for line in path.read_text().splitlines():
            if line.startswith("dram_bytes_per_vector:"):
                return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


# ---------------------------------------------------------------------------
# Arms
# ---------------------------------------------------------------------------
def reference_arm(args, rank: int, world: int) -> None:
    """The reference's FP64 path (oracle port) on the host cores: every core
    propagates its own trajectory of the benchmark system continuously over a
    ``--ref-horizon``-us prefix at the GPU arm's state-error budget (scaled by
    the prefix's share of the 5-us horizon, as the reference's full-size
    runner scales it), after a short warm-up prefix.  The timed prefix covers
    all ``steps`` (ms_per_step is its wall time / steps).  Trajectories/s
    extrapolate the prefix to 5-us trajectories and divide by the recorded
    ratio of a full 5-us run's time to that extrapolation
    (oracle/cpu_extrapolation.json), which raises the CPU figure."""
    if rank != 0:
        return
    from rpm_b200.autotune import budget_for_yield_tolerance

    budget = args.budget if args.budget is not None else budget_for_yield_tolerance(YIELD_TOL)
    base = CpuBaseline(cpu_workers(), budget)
    if args.warmup:
        base.segment(0.0025)
    mv0 = base.matvecs
    wall = base.segment(args.ref_horizon)
    base.close()
    raw = base.workers * (args.ref_horizon / HORIZON_US) / wall
    record = extrapolation_record()
    factor = None
    for row in (record or {}).get("summary") or []:
        if row.get("impl") == "port" and abs(row.get("budget", 0.0) - budget) <= 1e-12 * max(1.0, budget):
            factor = row.get("full_over_extrapolated")
    value = raw / factor if factor else raw
    cpu = {"value": value, "unit": UNIT, "cores": base.workers, "kind": "port",
           "why_port": "the reference is pure Python/NumPy and cannot travel to the GPU box; the port restates "
                       "its FP64 path (oracle/rpm_oracle.py); extrapolation.port_over_reference gives the port's "
                       "time relative to the reference's own code on one host",
           "sample": f"{base.workers} trajectories (one per core), each propagated continuously over a "
                     f"{args.ref_horizon:g}-us prefix at budget {budget:g} (the GPU arm's) scaled to the prefix, "
                     f"extrapolated to 5 us" + (f" and divided by the recorded full/extrapolated time ratio "
                                                f"{factor:.3f}" if factor else ""),
           "extrapolated_value": raw, "full_over_extrapolated": factor, "budget": budget,
           "prefix_us": args.ref_horizon, "matvecs": base.matvecs - mv0, "extrapolation": record}
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": {"workload": WORKLOAD, "state_error_budget": budget, "krylov": "adaptive 8-40 (reference controller)",
                   "parallelism": f"one trajectory per host core x{base.workers}"},
        "cpu_baseline": cpu,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def hpsi_probe(args) -> None:
    """Complex64 H psi alone: ``--hpsi-only K`` times K launches over
    orientations x vectors full-size states of one orientation (the batched
    step's H psi shape) and prints one diagnostic JSON line.  Used for kernel
    timing and as a short ncu target; not a benchmark line."""
    import torch

    import rpm_b200 as rb
    from rpm_b200 import _lib, synthetic

    full = synthetic.full_system()
    h = rb.CompiledFullPairHamiltonian(full.dimensions, full.terms(math.pi / 4, 0.0), left_axes=full.left_axes,
                                       right_axes=full.right_axes)
    n = full.dimension
    batch = args.orientations * args.vectors
    ld = (n + 63) // 64 * 64
    g = torch.Generator(device="cuda").manual_seed(5)
    x = torch.randn((batch, ld), dtype=torch.complex64, device="cuda", generator=g)
    y = torch.empty_like(x)

    def launch():
        _lib.call("rpm_hpsi", h._system.handle, _lib.PREC_C64, _lib.ptr(x), _lib.ptr(y), batch, ld,
                  _lib.stream_handle())

    for _ in range(max(3, args.warmup)):
        launch()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.hpsi_only):
        launch()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.hpsi_only
    peak, _ = measured_peak_hbm()
    gbs = 16.0 * n * batch / (ms * 1e-3) / 1e9
    print(json.dumps({"probe": "hpsi_c64", "vectors": batch, "n": n, "fast_kernels": h._system.fast_hpsi,
                      "ms_per_launch_pair": ms, "algorithmic_GBps": gbs, "hbm_frac": gbs / peak}), flush=True)


def adjoint_sample(full, direction, dev, vectors: int = 16, horizon_us: float = 1.0):
    """Yield gradients (|B|, theta, phi, pulse amplitude, hyperfine scale) of
    `vectors` random-phase trajectories of the full system with a 300 nT
    transverse pulse on [0.2, 0.7] us, timed forward + backward on the device
    for both adjoint precisions; a side measurement next to the main line."""
    import numpy as np
    import torch

    from rpm_b200 import adjoint, synthetic

    params = np.array([50.0, direction[0], direction[1], 300.0, 1.0])
    model = adjoint.ParametricRadicalPair(full, pulse_start_us=0.2, pulse_duration_us=0.5)
    times = np.arange(int(round(horizon_us / GRID_US)) + 1) * GRID_US
    states = list(synthetic.random_phase_vectors(full.dimensions, vectors, 4242))
    out = {"metric": "adjoint yield-gradient throughput, 5 parameters", "unit": "trajectory-us/s",
           "sample": f"{vectors} trajectories x {horizon_us:g} us (221,184 dims, 300 nT pulse on [0.2, 0.7] us)"}
    try:
        for precision in ("c128", "c64"):
            engine = adjoint.AdjointYieldGradient(model, precision=precision)
            torch.cuda.synchronize(dev)
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record()
            fwd = engine.forward(params, states, times, LIFETIME_US)
            e1.record()
            grads, diag = engine.backward(params, fwd)
            e2.record()
            torch.cuda.synchronize(dev)
            fwd["workspace"].close()
            total = e0.elapsed_time(e2) / 1e3
            out[precision] = {"value": vectors * horizon_us / total, "forward_s": e0.elapsed_time(e1) / 1e3,
                              "backward_s": e1.elapsed_time(e2) / 1e3, "taylor_degree": diag["taylor_degree"],
                              "max_taylor_tail": diag["max_taylor_tail"],
                              "checkpoint_drift": diag["checkpoint_drift"],
                              "mean_gradient": [float(v) for v in grads.mean(axis=0)]}
    except Exception as exc:  # a side measurement must not sink the main line
        out["error"] = f"{type(exc).__name__}: {exc}"
    return out


UNEVEN_COUNTS = {3: 512, 5: 320, 7: 192}  # nuclei per radical -> trajectories (864 / 13,824 / 221,184 dims)


def uneven_sample(args, scale: float = 1.0, horizon_us: float = HORIZON_US) -> dict:
    """Uneven system sizes with unequal recombination rates, mixed in every
    launch: equal-count nuclear prefixes of 3, 5 and 7 nuclei per radical (6,
    10 and 14 nuclei; 864, 13,824 and 221,184 dimensions), kS = 1e6 and
    kT = 2e6 s^-1, trajectories split 512 : 320 : 192 (times ``scale``), each
    with its own field direction drawn without repetition from a 64 x 32
    (theta, phi) grid at 50 uT and its own random-phase vector, to
    ``horizon_us``.  Each shape group is autotuned alone on a 0.25-us prefix
    (Krylov dimension 16-40 and tile, accuracy-gated); the group's dimension
    becomes its systems' Krylov cap in the mixed batch, and each launch
    carries at most one tile of every group.  Timed end to end through
    ``propagate`` (host states in, yields out); a tight-budget rerun of two
    trajectories per group at the batch's largest dimension checks the yields."""
    import numpy as np
    import torch

    import rpm_b200 as rb
    from rpm_b200 import synthetic
    from rpm_b200.autotune import KRYLOV_RANGE, tune_per_shape
    from rpm_b200.batched import BatchedPropagator

    full = synthetic.full_system()
    counts = {per: max(2, int(round(c * scale))) for per, c in UNEVEN_COUNTS.items()}
    grid = [(math.pi * (i + 0.5) / 64, 2 * math.pi * j / 32) for i in range(64) for j in range(32)]
    rng = np.random.default_rng(404)
    pick = rng.permutation(len(grid))
    hams, states, dims, group_pos = [], [], [], []
    t_setup = time.perf_counter()
    for per, count in counts.items():
        sub = synthetic.prefix_system(full, per) if per < 7 else full
        pos = []
        for _ in range(count):
            th, ph = grid[int(pick[len(hams) % len(grid)])]
            h = rb.CompiledFullPairHamiltonian(sub.dimensions, sub.terms(th, ph), left_axes=sub.left_axes,
                                               right_axes=sub.right_axes)
            h.set_recombination_rates(1.0, 2.0)
            pos.append(len(hams))
            hams.append(h)
            states.append(synthetic.random_phase_vectors(sub.dimensions, 1, 900 + len(states))[0])
            dims.append(sub.dimension)
        group_pos.append(pos)
    t_setup = time.perf_counter() - t_setup
    index = list(range(len(hams)))
    times = np.arange(int(round(horizon_us / GRID_US)) + 1) * GRID_US
    # tuning sample: up to 192 trajectories of every group
    sample = [p for pos in group_pos for p in pos[:192]]
    t_tune = time.perf_counter()
    tuning = tune_per_shape([hams[p] for p in sample], [states[p] for p in sample], list(range(len(sample))),
                            horizon_us=0.25, full_horizon_us=horizon_us, yield_tolerance=YIELD_TOL,
                            krylov_dimensions=KRYLOV_RANGE, tiles=(16, 48, 96, 192, 320, 512))
    t_tune = time.perf_counter() - t_tune
    group_caps = [r.krylov_dimension for r in tuning.results]
    group_tiles = [r.tile for r in tuning.results]
    caps = [group_caps[g] for g, pos in enumerate(group_pos) for _ in pos]
    bp = BatchedPropagator(hams, krylov_dimension=max(caps), state_error_budget=tuning.state_error_budget,
                           krylov_caps=caps)
    chunks = max(-(-len(pos) // t) for pos, t in zip(group_pos, group_tiles))
    launches = []
    for c in range(chunks):
        sel = []
        for pos in group_pos:
            per_chunk = -(-len(pos) // chunks)
            sel += pos[c * per_chunk:(c + 1) * per_chunk]
        launches.append(sel)
    first = [pos[0] for pos in group_pos]
    bp.propagate([states[k] for k in first], times[:9], system_index=first)  # warm-up
    torch.cuda.synchronize()
    yields = np.empty(len(hams))
    stats = [None] * len(hams)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for sel in launches:
        out = bp.propagate([states[k] for k in sel], times, system_index=sel)
        yields[sel] = out.yields
        for k, st in zip(sel, out.stats):
            stats[k] = st
    e1.record()
    torch.cuda.synchronize()
    seconds = e0.elapsed_time(e1) / 1e3
    # tight-budget check of two trajectories per group
    check = [p for pos in group_pos for p in pos[:2]]
    tight = BatchedPropagator([hams[k] for k in check], krylov_dimension=max(KRYLOV_RANGE),
                              state_error_budget=tuning.state_error_budget / 100.0).propagate(
        [states[k] for k in check], times, system_index=list(range(len(check))))
    err = np.abs(tight.yields - yields[check])
    per_group = []
    for g, pos in enumerate(group_pos):
        per_group.append({"dimension": dims[pos[0]], "trajectories": len(pos), "krylov_cap": group_caps[g],
                          "tile": group_tiles[g],
                          "accepted_steps_mean": float(np.mean([stats[k].accepted_steps for k in pos])),
                          "matvecs_mean": float(np.mean([stats[k].matvecs for k in pos])),
                          "yield_range": [float(yields[pos].min()), float(yields[pos].max())],
                          "tuned_throughput_traj_us_per_s": tuning.results[g].throughput})
    return {"workload": "uneven sizes 864 / 13,824 / 221,184 with kS = 1e6, kT = 2e6 s^-1 (Arnoldi), "
                        "64 x 32 direction grid, one launch mixes every size",
            "trajectories": len(hams), "horizon_us": float(times[-1]), "seconds": seconds,
            "trajectories_per_s": len(hams) / seconds, "launches": chunks, "timed": "propagate (host in, yields out)",
            "groups": per_group, "state_error_budget": tuning.state_error_budget,
            "yield_err_vs_tight_budget": {"max": float(err.max()), "trajectories": len(check)},
            "setup_s": t_setup, "tune_s": t_tune, "rates_per_us": [1.0, 2.0]}


def ncu_traffic_per_vector_iteration():
    """DRAM bytes per vector and Lanczos iteration of the persistent kernel
    from its committed ncu summary, or None."""
    path = ROOT / "profiles" / "lanczos_persistent_c64.md"
    try:
        for line in path.read_text().splitlines():
            if line.startswith("dram_bytes_per_vector_iteration:"):
                return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


BENCH_TILES = (8, 16, 24, 48)  # trajectories per propagate call (divisors of the 48-trajectory step)


def b200_arm(args, rank: int, world: int, dist) -> None:
    import numpy as np
    import torch

    import rpm_b200 as rb
    from rpm_b200 import synthetic
    from rpm_b200.autotune import KRYLOV_RANGE, budget_for_yield_tolerance, tune
    from rpm_b200.batched import BatchedPropagator
    from rpm_b200.distributed import gather_yields, max_over_ranks, rank_shard

    from rpm_b200 import _lib

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    _lib.call("rpm_set_persistent_warps", args.persistent_warps)
    _lib.call("rpm_set_gram_kernel", 1 if args.gram == "tensor" else 0)
    full = synthetic.full_system()
    dirs = synthetic.fibonacci_sphere(args.orientations)
    hams = [rb.CompiledFullPairHamiltonian(full.dimensions, full.terms(th, ph), left_axes=full.left_axes,
                                           right_axes=full.right_axes) for th, ph in dirs]
    n = full.dimension
    nvec = args.vectors
    per_rank = args.orientations * nvec
    # The whole job is world x (orientations x vectors) trajectories, the same
    # list on every rank; each rank propagates its cost-balanced shard of it.
    job = world * per_rank
    start, end = rank_shard([n] * job, dist)
    ntraj = end - start
    gids = np.arange(start, end)
    system_index = ((gids % per_rank) // nvec).astype(np.int32)
    states = np.stack([synthetic.random_phase_vectors(full.dimensions, 1, 1000 + int(g // per_rank) * 1000
                                                      + int(g % nvec))[0] for g in gids])
    times = np.arange(int(round(args.horizon / GRID_US)) + 1) * GRID_US
    tuning = None
    krylov, budget, reorth = args.krylov, args.budget, args.reorth_period
    tile = ntraj
    if budget is None:
        budget = budget_for_yield_tolerance(YIELD_TOL)
    if krylov == "auto":
        # Krylov cap over the batched configuration's range 16-40, tile over
        # divisors of the step's batch, reorthogonalisation none / every 16
        # iterations; only candidates within the yield accuracy gate compete
        tiles = tuple(t for t in BENCH_TILES if ntraj % t == 0) or (ntraj,)
        tuning = tune(hams, list(states), system_index, horizon_us=0.25, full_horizon_us=args.horizon,
                      yield_tolerance=YIELD_TOL, krylov_dimensions=KRYLOV_RANGE, tiles=tiles,
                      reorth_periods=(0, 16), lanczos_kernel=args.lanczos)
        krylov, tile, reorth = tuning.krylov_dimension, tuning.tile, tuning.reorth_period
    krylov = int(krylov)
    knobs = dict(krylov_dimension=krylov, state_error_budget=budget, lanczos_kernel=args.lanczos,
                 wavefront=args.wavefront, reorth_period=reorth)
    if args.parts > 1:
        # independent halves of the step on two streams: one half's controller,
        # Gram and rebuild run beside the other half's persistent Lanczos launch
        from rpm_b200.batched import ConcurrentBatches

        bp = ConcurrentBatches(hams, parts=args.parts, reserve_sms=args.reserve_sms, **knobs)
        tile = ntraj
    else:
        bp = BatchedPropagator(hams, **knobs)
    ld = bp.leading_dimension
    pristine = torch.zeros((ntraj, ld), dtype=torch.complex128, device=dev)
    pristine[:, :n].copy_(torch.from_numpy(states))
    work = torch.empty_like(pristine)
    chunks = [(a, min(a + tile, ntraj)) for a in range(0, ntraj, tile)]

    def step():
        work.copy_(pristine)
        values, stats = [], []
        for a, b in chunks:
            v, _, st = bp.propagate_device(work[a:b], times, system_index[a:b])
            values.append(v)
            stats.extend(st)
        return torch.cat(values), stats

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    bp.counters(reset=True)
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    clocks = ClockSampler(uuid)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_start.record()
    values = stats = None
    for _ in range(args.steps):
        values, stats = step()
    t_end.record()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clock_info = clocks.stop()
    elapsed = max_over_ranks(t_start.elapsed_time(t_end) / 1e3, dist, dev)
    counters = bp.counters(reset=True)
    kind = bp.lanczos_kind()
    value = args.steps * job / elapsed
    yields = bp.yields_device(times, values, LIFETIME_US)
    yields_all = gather_yields(yields, dist)  # the only cross-rank data: per-trajectory yields
    bad = [s.status for s in stats if s.status]
    if bad:
        raise RuntimeError(f"batched propagation failed with status {bad[0]}")

    # end-to-end through the public API from pinned host memory
    host_states = torch.from_numpy(states).pin_memory()
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    d2h = 0
    for _ in range(e2e_steps):
        d2h = 0
        for a, b in chunks:
            res = bp.propagate(host_states[a:b], times, system_index=system_index[a:b], lifetime_us=LIFETIME_US)
            d2h += res.observable_values.nbytes + res.state_error_estimates.nbytes + res.yields.nbytes
    e1.record()
    torch.cuda.synchronize()
    e2e_elapsed = max_over_ranks(e0.elapsed_time(e1) / 1e3, dist, dev)
    e2e_value = e2e_steps * job / e2e_elapsed
    h2d = ntraj * n * 16

    line = None
    if rank == 0:
        # roofline of the dominant kernel, timed live (CUDA events inside the
        # graph) on the first Krylov step of every propagate call: one
        # persistent launch runs all m Lanczos iterations of `tile`
        # trajectories, each iteration reading w'_j and v_{j-1} and writing v_j
        # and w'_{j+1} (32 N bytes per vector); the per-iteration pass pair
        # moves the same bytes
        peak, peak_src = measured_peak_hbm()
        iter_s = counters["hpsi_ms"] / 1e3
        persistent = kind == "persistent"
        iters = krylov if persistent else 1
        per_launch = tile // max(1, args.parts)  # trajectories of one launch
        alg_bytes = 32.0 * n * per_launch * iters
        launch_s = iter_s * iters
        achieved = alg_bytes / launch_s / 1e9 if launch_s > 0 else None
        per_vec_iter = ncu_traffic_per_vector_iteration() if persistent else ncu_traffic_per_vector(True)
        kernel = (f"k_lanczos_persistent<2,5,1,6> (all {krylov} Lanczos iterations of a Krylov step for {per_launch} "
                  "trajectories: complex64 H psi + Paige 3-term recurrence, TMA-staged)" if persistent else
                  "fast_pass_r + fast_pass_l (one fused Lanczos iteration, all trajectories)")
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak if achieved else None,
                    "traffic": per_vec_iter * per_launch * iters if per_vec_iter is not None else None,
                    "traffic_source": ("profiles/lanczos_persistent_c64.md (ncu capture of this kernel; command "
                                       "there), scaled to one launch" if persistent else
                                       "profiles/lanczos_iteration_fused_c64.md"),
                    "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs)" if peak_src == "measured" else "fallback",
                    "kernel": kernel, "algorithmic_bytes": alg_bytes, "avg_launch_ms": launch_s * 1e3,
                    "ms_per_lanczos_iteration": counters["hpsi_ms"], "samples": counters["hpsi_samples"]}
        # plain single-vector FP64 GPU path (config 1's drop-in), one
        # trajectory per orientation: its time, and the batched yield errors
        plain, y_err = None, None
        if not args.no_plain:
            errs, secs, mvs = [], 0.0, 0
            for k in range(min(args.plain_trajectories, args.orientations)):
                b = k * nvec  # orientation k, vector 0
                t0 = time.perf_counter()
                ref = rb.AdaptiveLanczosPropagator(hams[system_index[b]], minimum_dimension=8, maximum_dimension=40,
                                                   state_error_budget=1e-10).propagate(
                    states[b], times, rb.SingletPopulationObservable(full.dimensions))
                torch.cuda.synchronize()
                secs += time.perf_counter() - t0
                mvs += ref.stats.matvecs
                y_plain = rb.integrate_yield(times, ref.observable_values, LIFETIME_US)
                errs.append(abs(float(yields[b].item()) - y_plain))
            errs = np.asarray(errs)
            y_err = {"max": float(errs.max()), "rms": float(np.sqrt(np.mean(errs ** 2))), "trajectories": int(errs.size),
                     "per_orientation": [float(e) for e in errs]}
            plain = {"value": errs.size / secs, "unit": UNIT,
                     "sample": f"{errs.size} trajectories (vector 0 of each orientation), {args.horizon:g} us",
                     "matvecs": mvs, "krylov": "8-40", "budget": 1e-10}
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            base = CpuBaseline(cpu_workers(), budget)
            wall = base.segment(args.cpu_horizon)
            base.close()
            cpu = {"value": base.workers * (args.cpu_horizon / HORIZON_US) / wall, "unit": UNIT,
                   "cores": base.workers, "kind": "port",
                   "sample": f"{base.workers} trajectories (one per core) x {args.cpu_horizon:g} us prefix (Krylov "
                             f"8-40, budget {budget:g} scaled to the prefix), extrapolated to 5 us; {wall:.1f} s",
                   "extrapolation": extrapolation_record()}
        adjoint = None
        if world == 1 and not args.no_adjoint:
            adjoint = adjoint_sample(full, dirs[0], dev)
        uneven = None
        if world == 1 and not args.no_uneven:
            uneven = uneven_sample(args, args.uneven_scale)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64 H-psi/basis + f64 Krylov control", "data": "synthetic",
            "config": {"workload": WORKLOAD, "batch": f"{args.orientations} Fibonacci field orientations x {nvec} "
                                                      "random-phase vectors per GPU per step",
                       "trajectories_per_step_per_gpu": per_rank, "krylov_dim": krylov, "tile": tile,
                       "concurrent_parts": args.parts,
                       "reorth_period": reorth, "lanczos_kernel": kind, "gram_kernel": args.gram,
                       "tuning": ("autotuned: Krylov " + str(list(KRYLOV_RANGE)) + ", tile, reorthogonalisation "
                                  "(none / 16), accuracy-gated" if tuning else "fixed"),
                       "state_error_budget": budget, "parallelism": f"replicas x{world} (cost-balanced shards)",
                       "l2": "inputs larger than L2 (Krylov basis " f"{tile * (krylov + 1) * n * 8 / 1e9:.1f} GB)"},
            "autotune": ({"trials": tuning.trials, "horizon_us": 0.25, "budget_scaled_to_prefix": True}
                         if tuning else None),
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": e2e_steps},
            "gpu_launches": counters["kernel_launches"],
            "clocks": clock_info,
            "plain_fp64": plain,
            "batched_over_plain": value / world / plain["value"] if plain else None,
            "yield_err_vs_fp64": y_err,
            "yields_gathered": int(yields_all.numel()),
            "adjoint": adjoint,
            "uneven_sizes": uneven,
        }
    if line is not None:
        print(json.dumps(line), flush=True)


def main() -> None:
    p = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=8)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=("b200", "reference"), default="b200")
    p.add_argument("--orientations", type=int, default=12)
    p.add_argument("--vectors", type=int, default=4, help="random-phase vectors per orientation per GPU")
    p.add_argument("--krylov", default="auto", help="Krylov dimension, or 'auto' (autotuned over 16-40)")
    p.add_argument("--budget", type=float, default=None,
                   help="accumulated state-error budget (default: half the 1e-6 yield tolerance)")
    p.add_argument("--e2e-steps", type=int, default=2)
    p.add_argument("--lanczos", choices=("persistent", "passes"), default="persistent",
                   help="Lanczos iterations of a Krylov step: one persistent launch, or two pass launches each")
    p.add_argument("--wavefront", type=int, default=0, help="persistent kernel: vectors per wavefront group (0: equal groups of at most 16)")
    p.add_argument("--parts", type=int, default=1,
                   help="run the step's trajectories as this many concurrent batches on their own streams")
    p.add_argument("--reserve-sms", type=int, default=16,
                   help="with --parts > 1: SMs each persistent launch leaves to the other batch's kernels")
    p.add_argument("--gram", choices=("tensor", "cuda"), default="tensor",
                   help="singlet Gram kernel: tcgen05 tensor cores or CUDA cores")
    p.add_argument("--persistent-warps", type=int, choices=(8, 9, 10), default=8,
                   help="persistent kernel: consumer warps per CTA")
    p.add_argument("--reorth-period", type=int, default=0,
                   help="reorthogonalise the next Lanczos vector every this many iterations (0: never)")
    p.add_argument("--cpu-horizon", type=float, default=0.05, help="us of the GPU arm's CPU baseline sample")
    p.add_argument("--ref-horizon", type=float, default=0.25,
                   help="reference arm: us of every host trajectory covered by the timed steps")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-plain", action="store_true", help="skip the plain FP64 comparison trajectories")
    p.add_argument("--plain-trajectories", type=int, default=12,
                   help="plain FP64 trajectories (vector 0 of that many orientations) for the yield errors")
    p.add_argument("--no-adjoint", action="store_true", help="skip the adjoint-gradient side measurement")
    p.add_argument("--uneven", action="store_true",
                   help="only the uneven-size side measurement (864 / 13,824 / 221,184 with unequal rates)")
    p.add_argument("--uneven-scale", type=float, default=1.0,
                   help="uneven-size side measurement: trajectory counts as a fraction of 512 / 320 / 192")
    p.add_argument("--no-uneven", action="store_true", help="skip the uneven-size side measurement")
    p.add_argument("--adjoint-only", action="store_true",
                   help="diagnostic: only the adjoint side measurement (--vectors trajectories, --horizon us)")
    p.add_argument("--horizon", type=float, default=HORIZON_US,
                   help="propagation horizon in us (5 us is the benchmark workload; shorter only for profiling)")
    p.add_argument("--hpsi-only", type=int, default=0, metavar="K",
                   help="diagnostic: time K complex64 H psi launches over orientations x vectors states and exit")
    args = p.parse_args()
    if args.warmup < 0 or args.steps < 1:
        raise SystemExit("steps must be >= 1 and warmup >= 0")
    if args.hpsi_only > 0:
        hpsi_probe(args)
        return
    if args.uneven:
        print(json.dumps(uneven_sample(args, args.uneven_scale, args.horizon)), flush=True)
        return
    if args.adjoint_only:
        import torch

        from rpm_b200 import synthetic

        full = synthetic.full_system()
        out = adjoint_sample(full, synthetic.fibonacci_sphere(args.orientations)[0], torch.device("cuda", 0),
                             vectors=args.vectors, horizon_us=args.horizon)
        print(json.dumps(out), flush=True)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist_mod

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        backend = "nccl" if args.impl == "b200" else "gloo"
        dist_mod.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        dist = dist_mod
    try:
        if args.impl == "reference":
            reference_arm(args, rank, world)
        else:
            b200_arm(args, rank, world, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
