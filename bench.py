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


# ---------------------------------------------------------------------------
# CPU baseline (oracle port), run in spawned worker processes
# ---------------------------------------------------------------------------
_CPU_STATE = {}


def _cpu_worker_init():
    import oracle
    from rpm_b200 import synthetic

    full = synthetic.full_system()
    terms = full.terms(math.pi / 4, 0.0)
    h = oracle.CompiledFullPairHamiltonian(full.dimensions, [oracle.LocalTerm(t.axes, t.operator) for t in terms],
                                           left_axes=full.left_axes, right_axes=full.right_axes)
    _CPU_STATE["h"] = h
    _CPU_STATE["dims"] = full.dimensions


def _cpu_worker_run(args):
    seed, horizon = args
    import numpy as np

    import oracle
    from rpm_b200 import synthetic

    h = _CPU_STATE["h"]
    psi = synthetic.random_phase_vectors(_CPU_STATE["dims"], 1, seed)[0]
    times = np.arange(int(round(horizon / GRID_US)) + 1) * GRID_US
    prop = oracle.AdaptiveLanczosPropagator(h, minimum_dimension=8, maximum_dimension=40,
                                            state_error_budget=1e-10 * horizon / HORIZON_US)
    t0 = time.perf_counter()
    res = prop.propagate(psi, times, oracle.SingletPopulationObservable(_CPU_STATE["dims"]))
    return time.perf_counter() - t0, res.stats.matvecs


class CpuBaseline:
    """The oracle's FP64 port on `workers` host processes (one BLAS thread each)."""

    def __init__(self, workers: int):
        import multiprocessing as mp

        for var in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
            os.environ[var] = "1"
        self.workers = workers
        self.pool = mp.get_context("spawn").Pool(workers, initializer=_cpu_worker_init)

    def round(self, horizon: float, seed0: int):
        """One round: every worker propagates one trajectory over `horizon` us."""
        t0 = time.perf_counter()
        out = self.pool.map(_cpu_worker_run, [(seed0 + k, horizon) for k in range(self.workers)])
        wall = time.perf_counter() - t0
        per_traj = sum(o[0] for o in out) / len(out)
        # trajectories/s over the full horizon, all workers in parallel
        return self.workers / (wall * HORIZON_US / horizon), per_traj, wall

    def close(self):
        self.pool.close()
        self.pool.join()


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
    if rank != 0:
        return
    base = CpuBaseline(cpu_workers())
    horizon = args.cpu_horizon
    for k in range(args.warmup):
        base.round(horizon, 1000 + 64 * k)
    vals = []
    t0 = time.perf_counter()
    for k in range(args.steps):
        v, _, _ = base.round(horizon, 5000 + 64 * k)
        vals.append(v)
    wall = time.perf_counter() - t0
    base.close()
    value = sum(vals) / len(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * wall / max(1, args.steps), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": {"workload": "plain FP64 Lanczos (Krylov 8-40, budget 1e-10) on the 221,184-dim synthetic "
                               "radical pair, theta = pi/4, one trajectory per host core, extrapolated from a "
                               f"{horizon} us prefix to 5 us"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": base.workers, "kind": "port",
                         "sample": f"each step: {base.workers} trajectories x {horizon} us prefix, extrapolated"},
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


def uneven_sample(args) -> dict:
    """Uneven system sizes with unequal recombination rates in one propagate
    call: equal-count nuclear prefixes of 3, 5 and 7 nuclei per radical (864,
    13,824 and 221,184 dimensions), kS = 1e6 and kT = 2e6 s^-1, trajectories
    split 16 : 10 : 6 (the 512 : 320 : 192 proportions at 1/32 scale), field
    directions from a 64 x 32 (theta, phi) grid, Arnoldi per shape group."""
    import numpy as np
    import torch

    import rpm_b200 as rb
    from rpm_b200 import synthetic
    from rpm_b200.batched import BatchedPropagator

    full = synthetic.full_system()
    counts = {3: 16, 5: 10, 7: 6}
    grid = [(math.pi * (i + 0.5) / 64, 2 * math.pi * j / 32) for i in range(64) for j in range(32)]
    rng = np.random.default_rng(404)
    hams, states, index, dims = [], [], [], []
    for per, count in counts.items():
        sub = synthetic.prefix_system(full, per) if per < 7 else full
        for t in range(count):
            th, ph = grid[int(rng.integers(len(grid)))]
            h = rb.CompiledFullPairHamiltonian(sub.dimensions, sub.terms(th, ph), left_axes=sub.left_axes,
                                               right_axes=sub.right_axes)
            h.set_recombination_rates(1.0, 2.0)
            index.append(len(hams))
            hams.append(h)
            states.append(synthetic.random_phase_vectors(sub.dimensions, 1, 900 + len(states))[0])
            dims.append(sub.dimension)
    times = np.arange(int(round(args.horizon / GRID_US)) + 1) * GRID_US
    from rpm_b200.autotune import KRYLOV_RANGE, tune

    tuning = tune(hams, states, index, horizon_us=0.25, yield_tolerance=YIELD_TOL, krylov_dimensions=KRYLOV_RANGE,
                  tiles=(len(states),))
    bp = BatchedPropagator(hams, krylov_dimension=tuning.krylov_dimension, state_error_budget=0.5 * YIELD_TOL)
    first = [0, counts[3], counts[3] + counts[5]]  # one trajectory of each size
    bp.propagate([states[k] for k in first], times[:9], system_index=first)  # warm-up
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    out = bp.propagate(states, times, system_index=index)
    e1.record()
    torch.cuda.synchronize()
    seconds = e0.elapsed_time(e1) / 1e3
    return {"probe": "uneven_sizes_unequal_rates", "trajectories": len(states), "seconds": seconds,
            "trajectories_per_s": len(states) / seconds, "horizon_us": float(times[-1]),
            "dimensions": {str(d): dims.count(d) for d in sorted(set(dims))},
            "yield_range": [float(np.min(out.yields)), float(np.max(out.yields))],
            "krylov_dim": tuning.krylov_dimension,
            "autotune": [{k: t[k] for k in ("krylov_dimension", "throughput") if k in t} for t in tuning.trials],
            "rates_per_us": [1.0, 2.0]}


def b200_arm(args, rank: int, world: int, dist) -> None:
    import numpy as np
    import torch

    import rpm_b200 as rb
    from rpm_b200 import synthetic
    from rpm_b200.batched import BatchedPropagator
    from rpm_b200.distributed import gather_yields, max_over_ranks

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    full = synthetic.full_system()
    dirs = synthetic.fibonacci_sphere(args.orientations)
    hams = [rb.CompiledFullPairHamiltonian(full.dimensions, full.terms(th, ph), left_axes=full.left_axes,
                                           right_axes=full.right_axes) for th, ph in dirs]
    n = full.dimension
    nvec = args.vectors
    ntraj = args.orientations * nvec
    seed = 1000 + rank
    vecs = synthetic.random_phase_vectors(full.dimensions, nvec, seed)
    states = np.stack([vecs[v] for k in range(args.orientations) for v in range(nvec)])
    system_index = np.array([k for k in range(args.orientations) for _ in range(nvec)], dtype=np.int32)
    times = np.arange(int(round(args.horizon / GRID_US)) + 1) * GRID_US
    tuning = None
    krylov, budget = args.krylov, args.budget
    if krylov == "auto" or budget is None:
        # Krylov dimension over the batched configuration's range 16-40 (tile
        # fixed at this workload's batch), budget from the yield tolerance
        from rpm_b200.autotune import KRYLOV_RANGE, budget_for_yield_tolerance, tune

        if krylov == "auto":
            tuning = tune(hams, list(states), system_index, horizon_us=0.25, yield_tolerance=YIELD_TOL,
                          krylov_dimensions=KRYLOV_RANGE, tiles=(ntraj,))
            krylov = tuning.krylov_dimension
        if budget is None:
            budget = budget_for_yield_tolerance(YIELD_TOL)
    krylov = int(krylov)
    bp = BatchedPropagator(hams, krylov_dimension=krylov, state_error_budget=budget)
    ld = bp.leading_dimension
    pristine = torch.zeros((ntraj, ld), dtype=torch.complex128, device=dev)
    pristine[:, :n].copy_(torch.from_numpy(states))
    work = torch.empty_like(pristine)

    def step():
        work.copy_(pristine)
        values, _, stats = bp.propagate_device(work, times, system_index)
        return values, stats

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
    value = args.steps * ntraj * world / elapsed
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
    for _ in range(e2e_steps):
        res = bp.propagate(host_states, times, system_index=system_index, lifetime_us=LIFETIME_US)
    e1.record()
    torch.cuda.synchronize()
    e2e_elapsed = max_over_ranks(e0.elapsed_time(e1) / 1e3, dist, dev)
    e2e_value = e2e_steps * ntraj * world / e2e_elapsed
    h2d = ntraj * n * 16
    d2h = res.observable_values.nbytes + res.state_error_estimates.nbytes + res.yields.nbytes

    line = None
    if rank == 0:
        # roofline of the dominant kernel pair, timed live on iteration 1 of
        # every Krylov step: with the shape-specialised passes one fused
        # Lanczos iteration (read w'_j and v_{j-1}, write v_j and w'_{j+1}:
        # 32 N bytes per vector), else one H psi (read psi, write H psi: 16 N)
        fused = bool(hams[0]._system.fast_hpsi)
        peak, peak_src = measured_peak_hbm()
        hpsi_s = counters["hpsi_ms"] / 1e3
        alg_bytes = (32.0 if fused else 16.0) * n * ntraj
        achieved = alg_bytes / hpsi_s / 1e9 if hpsi_s > 0 else None
        per_vec = ncu_traffic_per_vector(fused)
        kernel = ("fast_pass_r + fast_pass_l (one fused Lanczos iteration: complex64 H psi + Paige 3-term "
                  "recurrence, all trajectories)" if fused else
                  "cube_pass_l + cube_pass_r (complex64 H psi, one batched launch pair)")
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak if achieved else None,
                    "traffic": per_vec * ntraj if per_vec is not None else None,
                    "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs)" if peak_src == "measured" else "fallback",
                    "kernel": kernel, "algorithmic_bytes": alg_bytes, "avg_launch_ms": counters["hpsi_ms"],
                    "samples": counters["hpsi_samples"]}
        # plain single-vector FP64 GPU path on trajectory 0 (same state and system)
        plain, y_err = None, None
        if not args.no_plain:
            t0 = time.perf_counter()
            ref = rb.AdaptiveLanczosPropagator(hams[0], minimum_dimension=8, maximum_dimension=40,
                                               state_error_budget=1e-10).propagate(
                states[0], times, rb.SingletPopulationObservable(full.dimensions))
            torch.cuda.synchronize()
            plain_s = time.perf_counter() - t0
            y_plain = rb.integrate_yield(times, ref.observable_values, LIFETIME_US)
            y_err = abs(float(yields[0].item()) - y_plain)
            plain = {"value": 1.0 / plain_s, "unit": UNIT,
                     "sample": f"1 trajectory (orientation 0, vector 0), {args.horizon:g} us",
                     "matvecs": ref.stats.matvecs, "krylov": "8-40", "budget": 1e-10}
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            base = CpuBaseline(cpu_workers())
            cpu_value, per_traj, wall = base.round(args.cpu_horizon, 77)
            base.close()
            cpu = {"value": cpu_value, "unit": UNIT, "cores": base.workers, "kind": "port",
                   "sample": f"{base.workers} trajectories x {args.cpu_horizon} us prefix (Krylov 8-40, budget "
                             f"1e-10 scaled), extrapolated to 5 us; {per_traj:.1f} s each"}
        adjoint = None
        if world == 1 and not args.no_adjoint:
            adjoint = adjoint_sample(full, dirs[0], dev)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64 H-psi/basis + f64 Krylov control", "data": "synthetic",
            "config": {"workload": f"batched mixed-precision propagation, 221,184-dim synthetic FAD-TrpH-shaped radical "
                                   f"pair (2 e + 11 spin-1/2 + 3 spin-1), {args.orientations} Fibonacci field "
                                   f"orientations x {nvec} random-phase vectors per GPU per step, {args.horizon:g} us, "
                                   f"0.00125-us grid ({len(times)} points), singlet yield tau = 1 us",
                       "trajectories_per_step_per_gpu": ntraj, "krylov_dim": krylov,
                       "krylov_choice": ("autotuned over " + str([t["krylov_dimension"] for t in tuning.trials])
                                         if tuning else "fixed"),
                       "state_error_budget": budget, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (Krylov basis " f"{ntraj * (krylov + 1) * n * 8 / 1e9:.1f} GB)"},
            "autotune": ({"trials": [{k: t[k] for k in ("krylov_dimension", "throughput") if k in t}
                                     for t in tuning.trials], "horizon_us": 0.25} if tuning else None),
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
    p.add_argument("--cpu-horizon", type=float, default=0.025, help="us of the CPU baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-plain", action="store_true", help="skip the plain FP64 comparison trajectory")
    p.add_argument("--no-adjoint", action="store_true", help="skip the adjoint-gradient side measurement")
    p.add_argument("--uneven", action="store_true",
                   help="diagnostic: uneven sizes (864 / 13,824 / 221,184) with unequal rates, --horizon us")
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
        print(json.dumps(uneven_sample(args)), flush=True)
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
