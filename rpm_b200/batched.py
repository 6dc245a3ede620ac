"""Batched mixed-precision propagation of many radical-pair trajectories.

The batched counterpart of ``AdaptiveLanczosPropagator.propagate`` with the
singlet observable (``rpm_statevector_engine.py:717-933``): every trajectory
(state vector x system, where systems may differ in field orientation or bath
size) advances through its own adaptive Krylov steps, all of them inside one
fixed sequence of GPU launches per Krylov step that is replayed from a CUDA
graph.  The Krylov basis and H psi are complex64; alpha/beta, the state
between steps, the tridiagonal exponential, the error control, the singlet
Gram and populations and the Simpson yield are FP64.

Differences from the reference controller (the batched path is held to its
yields against the FP64 path, not to the reference's step decisions): the
Krylov dimension is fixed, and instead of
halving rejected steps, the step is the largest one whose embedded error
estimate meets the budget for that basis -- the basis does not depend on the
step, so no Krylov work is ever discarded.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _lib
from .engine import MatrixFreeHamiltonian, PropagationStats, _torch, population_bounds


@dataclass(frozen=True)
class BatchedResult:
    times_us: np.ndarray
    observable_values: np.ndarray        # (trajectories, times) singlet population
    observable_error_bounds: np.ndarray  # min(1, 2 eps + eps^2)
    state_error_estimates: np.ndarray
    yields: np.ndarray | None            # Simpson yield per trajectory (lifetime given)
    final_states: object | None          # (trajectories, N) complex128 CUDA tensor
    stats: tuple[PropagationStats, ...]
    status: np.ndarray


STATUS_TEXT = {
    1: "zero or non-finite initial state",
    2: "tridiagonal eigen-solver did not converge",
    3: "Lanczos step fell below the configured minimum.",
    4: "non-finite state",
}


class BatchedPropagator:
    """Propagate many trajectories of one or more Hamiltonians together.

    ``hamiltonians`` are rpm_b200 Hamiltonians with a radical split (for
    example from :func:`rpm_b200.build_hamiltonian` or a
    :class:`CompiledFullPairHamiltonian`); they may differ in dimension.

    ``lanczos_kernel``: "persistent" runs all Lanczos iterations of a Krylov
    step in one launch per shape group where the shape has a persistent
    kernel (else the per-iteration passes); "passes" launches the two
    shape-specialised passes per iteration.  ``wavefront``: vectors that move
    through the iterations together in the persistent kernel (0: equal groups
    of at most 16).
    ``reorth_period`` > 0 reorthogonalises the next Lanczos vector against the
    whole basis after every that many iterations (two classical Gram-Schmidt
    passes in FP64 over the complex64 basis); 0 keeps the plain three-term
    recurrence.  ``persistent_ctas`` > 0 limits a persistent launch to that
    many CTAs (one per SM otherwise), leaving SMs to another batch that runs
    concurrently on its own stream.  ``krylov_caps`` gives each Hamiltonian
    its own Krylov dimension (<= ``krylov_dimension``; 0 keeps the batch's),
    e.g. per system size in an uneven batch.
    """

    def __init__(self, hamiltonians: Sequence[MatrixFreeHamiltonian], *, krylov_dimension: int = 32,
                 embedded_offset: int = 4, safety_factor: float = 2.0, state_error_budget: float = 1e-7,
                 initial_step_us: float = 0.05, maximum_step_us: float = 0.25, minimum_step_us: float = 1e-9,
                 breakdown_relative: float = 1e-5, use_graph: bool = True, max_steps: int = 0,
                 lanczos_kernel: str = "persistent", wavefront: int = 0, reorth_period: int = 0,
                 persistent_ctas: int = 0, krylov_caps: Sequence[int] | None = None) -> None:
        hams = list(hamiltonians)
        if not hams:
            raise ValueError("At least one Hamiltonian is required.")
        for h in hams:
            if not isinstance(h, MatrixFreeHamiltonian) or not h._system.split:
                raise ValueError("the batched path needs rpm_b200 Hamiltonians with a radical split")
        self.hamiltonians = hams
        cfg = _lib.rpm_batch_config()
        cfg.krylov_dim = int(krylov_dimension)
        cfg.embedded_offset = int(embedded_offset)
        cfg.safety_factor = float(safety_factor)
        cfg.state_error_budget = float(state_error_budget)
        cfg.initial_step_us = float(initial_step_us)
        cfg.maximum_step_us = float(maximum_step_us)
        cfg.minimum_step_us = float(minimum_step_us)
        cfg.breakdown_relative = float(breakdown_relative)
        cfg.use_graph = 1 if use_graph else 0
        cfg.max_steps = int(max_steps)
        if lanczos_kernel not in ("persistent", "passes"):
            raise ValueError("lanczos_kernel must be 'persistent' or 'passes'")
        cfg.lanczos_kernel = 0 if lanczos_kernel == "persistent" else 1
        cfg.wavefront = int(wavefront)
        if int(reorth_period) < 0:
            raise ValueError("reorth_period must be >= 0")
        cfg.reorth_policy = 1 if int(reorth_period) > 0 else 0
        cfg.reorth_period = int(reorth_period)
        cfg.persistent_ctas = int(persistent_ctas)
        self.config = cfg
        handles = (ctypes.c_void_p * len(hams))(*[h._system.handle.value for h in hams])
        handle = ctypes.c_void_p()
        _lib.call("rpm_batch_create", handles, len(hams), ctypes.byref(cfg), ctypes.byref(handle))
        self._handle = handle
        ld = ctypes.c_longlong()
        _lib.call("rpm_batch_leading_dimension", handle, ctypes.byref(ld))
        self.leading_dimension = ld.value
        if krylov_caps is not None:
            caps = np.ascontiguousarray(krylov_caps, dtype=np.int32)
            if caps.size != len(hams):
                raise ValueError("krylov_caps needs one entry per Hamiltonian")
            _lib.call("rpm_batch_set_krylov_caps", handle, _lib.iptr(caps), int(caps.size))

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                _lib.call("rpm_batch_destroy", h)
            except Exception:
                pass
            self._handle = None

    def load_states(self, initial_states, system_index: Sequence[int]):
        """(trajectories, ld) complex128 CUDA buffer holding the initial states."""
        torch = _torch()
        idx = np.asarray(system_index, dtype=np.int32)
        ntraj = idx.size
        buf = torch.zeros((ntraj, self.leading_dimension), dtype=torch.complex128, device="cuda")
        sizes = {self.hamiltonians[k].dimension for k in idx}
        if isinstance(initial_states, (torch.Tensor, np.ndarray)) and initial_states.ndim == 2 and len(sizes) == 1:
            n = sizes.pop()
            if initial_states.shape[1] < n:
                raise ValueError("Initial state dimension does not match the Hamiltonian.")
            src = initial_states if isinstance(initial_states, torch.Tensor) else torch.from_numpy(
                np.ascontiguousarray(initial_states, dtype=np.complex128))
            # one copy for the whole batch (asynchronous from pinned host memory)
            buf[:, :n].copy_(src[:, :n], non_blocking=True)
            return buf
        for b in range(ntraj):
            n = self.hamiltonians[idx[b]].dimension
            row = initial_states[b]
            src = row if isinstance(row, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(row, dtype=np.complex128))
            if src.numel() < n:
                raise ValueError("Initial state dimension does not match the Hamiltonian.")
            buf[b, :n].copy_(src.reshape(-1)[:n])
        return buf

    def shape_order(self, system_index):
        """A stable order that puts trajectories of systems with the same shape
        (dimensions and radical split) next to each other, or None when they
        already are.  ``propagate_device`` launches H psi once per run of one
        shape, on the shape-specialised passes where the shape allows."""
        keys = {}
        for h in self.hamiltonians:
            keys.setdefault((tuple(h.dimensions), tuple(getattr(h, "left_axes", ()))), len(keys))
        shape = np.array([keys[(tuple(self.hamiltonians[k].dimensions),
                                tuple(getattr(self.hamiltonians[k], "left_axes", ())))] for k in system_index])
        runs = 1 + int(np.count_nonzero(np.diff(shape))) if shape.size else 0
        if runs <= len(np.unique(shape)):
            return None
        return np.argsort(shape, kind="stable")

    def propagate_device(self, psi, times_us, system_index, *, stream=None):
        """Run on a prepared (trajectories, ld) complex128 CUDA buffer (overwritten
        with the final states).  Returns device tensors (values, state_errors)
        and the per-trajectory ``rpm_batch_stats`` array."""
        torch = _torch()
        times = np.ascontiguousarray(times_us, dtype=np.float64)
        idx = np.ascontiguousarray(system_index, dtype=np.int32)
        ntraj = idx.size
        values = torch.empty((ntraj, times.size), dtype=torch.float64, device="cuda")
        errs = torch.empty_like(values)
        stats = (_lib.rpm_batch_stats * ntraj)()
        _lib.call("rpm_batch_propagate", self._handle, ntraj, _lib.iptr(idx), _lib.ptr(psi), _lib.dptr(times),
                  int(times.size), _lib.ptr(values), _lib.ptr(errs), stats, _lib.stream_handle(stream))
        return values, errs, stats

    def set_state_error_budget(self, budget: float) -> None:
        """Budget of later propagate calls (ENG:620-649 keeps it mutable too)."""
        _lib.call("rpm_batch_set_budget", self._handle, float(budget))

    def counters(self, reset: bool = False) -> dict:
        """Kernel launches, Krylov-step replays and the mean batched H psi time (ms)."""
        k, r, n = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        ms = ctypes.c_double()
        _lib.call("rpm_batch_counters", self._handle, 1 if reset else 0, ctypes.byref(k), ctypes.byref(r),
                  ctypes.byref(ms), ctypes.byref(n))
        return {"kernel_launches": k.value, "step_replays": r.value, "hpsi_ms": ms.value, "hpsi_samples": n.value}

    def lanczos_kind(self) -> str:
        """How the last propagation ran its Lanczos iterations: "persistent"
        (one launch per Krylov step and shape group), "passes" (two
        shape-specialised launches per iteration) or "cube" (general kernels)."""
        k = ctypes.c_int()
        _lib.call("rpm_batch_lanczos_kind", self._handle, ctypes.byref(k))
        return ("persistent", "passes", "cube")[k.value]

    def yields_device(self, times_us, values, lifetime_us: float):
        """Simpson yields of each row of ``values`` on the GPU (FP64, compensated)."""
        torch = _torch()
        t = torch.as_tensor(np.ascontiguousarray(times_us, dtype=np.float64), device="cuda")
        out = torch.empty(values.shape[0], dtype=torch.float64, device="cuda")
        _lib.call("rpm_simpson_yield", _lib.ptr(t), _lib.ptr(values), int(t.numel()), int(values.shape[0]),
                  int(values.shape[1]), float(lifetime_us), _lib.ptr(out), _lib.stream_handle())
        return out

    def recombination(self):
        """(kS, kT) shared by the batch's systems, or None (Hermitian propagation)."""
        rates = {h.recombination_rates for h in self.hamiltonians}
        if rates == {None}:
            return None
        if len(rates) != 1:
            raise ValueError("all systems of a batch must have the same recombination rates")
        return rates.pop()

    def propagate(self, initial_states, times_us, *, system_index: Sequence[int] | None = None,
                  lifetime_us: float | None = None, return_final_states: bool = False) -> BatchedResult:
        times = np.asarray(tuple(float(v) for v in times_us), dtype=float)
        if times.ndim != 1 or times.size == 0:
            raise ValueError("At least one observation time is required.")
        if np.any(times < 0.0) or np.any(np.diff(times) <= 0.0):
            raise ValueError("Observation times must be nonnegative and strictly increasing.")
        ntraj = len(initial_states)
        idx = np.zeros(ntraj, dtype=np.int32) if system_index is None else np.asarray(system_index, dtype=np.int32)
        if idx.size != ntraj:
            raise ValueError("system_index must give one system per trajectory")
        # trajectories of one shape run as one launch group: order them by shape
        order = self.shape_order(idx)
        states = initial_states if order is None else [initial_states[k] for k in order]
        run_idx = idx if order is None else idx[order]
        psi = self.load_states(states, run_idx)
        values, errs, stats = self.propagate_device(psi, times, run_idx)
        if order is not None:
            inverse = np.empty_like(order)
            inverse[order] = np.arange(order.size)
            torch = _torch()
            inv_t = torch.as_tensor(inverse, device=values.device)
            values, errs, psi = values[inv_t], errs[inv_t], psi[inv_t]
            stats = [stats[int(k)] for k in inverse]
        yields = None
        rates = self.recombination()
        if rates is not None:
            # singlet yield kS * int exp(-k_min t) P_S dt = (kS / k_min) * Simpson yield at tau = 1 / k_min
            if lifetime_us is not None:
                raise ValueError("with recombination rates the yield follows from the rates; omit lifetime_us")
            k_min = min(rates)
            if not k_min > 0.0:
                raise ValueError("the smaller recombination rate must be positive for a yield")
            yields = (rates[0] / k_min) * self.yields_device(times, values, 1.0 / k_min).cpu().numpy()
        elif lifetime_us is not None:
            yields = self.yields_device(times, values, lifetime_us).cpu().numpy()
        vals = values.cpu().numpy()
        se = errs.cpu().numpy()
        bounds = population_bounds(se) if se.size else se
        status = np.array([s.status for s in stats], dtype=np.int32)
        st = tuple(PropagationStats(s.accepted_steps, s.rejected_steps, int(s.matvecs), s.maximum_krylov_dimension,
                                    s.minimum_step_us, s.maximum_step_us, s.accumulated_state_error,
                                    s.maximum_norm_error) for s in stats)
        bad = [int(v) for v in status if v]
        if bad:
            raise RuntimeError(STATUS_TEXT.get(bad[0], f"batched propagation failed (status {bad[0]})"))
        return BatchedResult(times, vals, bounds, se, yields, psi if return_final_states else None, st, status)


@dataclass(frozen=True)
class BatchedSegment:
    """One segment of a batched segment propagation: trajectory b evolves under
    ``hamiltonians[system_index[b]]`` until ``end_us``; then ``pulse``
    (``(axis, unitary)`` or None) is applied to every trajectory unless
    ``end_us`` is the final time."""

    end_us: float
    hamiltonians: Sequence
    system_index: Sequence[int]
    pulse: tuple | None = None


def propagate_segments_batched(initial_states, times_us, segments: Sequence[BatchedSegment], *,
                               state_error_budget: float = 5e-7, lifetime_us: float | None = None,
                               krylov_dimension: int = 32, **knobs) -> BatchedResult:
    """Batched counterpart of :func:`rpm_b200.segments.propagate_segments`.

    Mirrors the reference's pulsed-control loop
    (``rpm_nuclear_spin_rotation_control.py:281-308``) for many trajectories at
    once: the horizon is cut at the segment ends; each segment runs the batched
    propagator with that segment's systems over the observation times inside
    it (shifted to start at the segment's start) with the budget scaled by the
    segment's duration; observation points carry the errors accumulated by
    earlier segments; between segments an instantaneous d x d unitary acts on
    one tensor axis of every state on the GPU.  A segment's systems may differ
    per trajectory (e.g. a field pulse of a per-trajectory amplitude); all
    segments must give each trajectory systems of the same dimensions.
    """
    torch = _torch()
    times = np.asarray(times_us, dtype=float)
    if times.ndim != 1 or times.size == 0 or times[0] != 0.0 or np.any(np.diff(times) <= 0.0):
        raise ValueError("Observation times must start at 0 and be strictly increasing.")
    segs = list(segments)
    if not segs or abs(segs[-1].end_us - times[-1]) > 1e-12:
        raise ValueError("The last segment must end at the final observation time.")
    ends = [s.end_us for s in segs]
    if any(b <= a for a, b in zip(ends, ends[1:])) or ends[0] <= 0.0:
        raise ValueError("Segment end times must be positive and strictly increasing.")
    ntraj = len(initial_states)
    for s in segs:
        if len(s.system_index) != ntraj:
            raise ValueError("every segment needs one system index per trajectory")
    def budget_of(k: int) -> float:
        start = 0.0 if k == 0 else float(segs[k - 1].end_us)
        return state_error_budget * (float(segs[k].end_us) - start) / times[-1]

    first = BatchedPropagator(segs[0].hamiltonians, krylov_dimension=krylov_dimension,
                              state_error_budget=budget_of(0), **knobs)
    idx0 = np.asarray(segs[0].system_index, dtype=np.int32)
    psi = first.load_states(initial_states, idx0)
    ld = first.leading_dimension
    dims = segs[0].hamiltonians[int(idx0[0])].dimensions
    n = int(np.prod(dims))
    values = np.empty((ntraj, times.size))
    errors = np.empty((ntraj, times.size))
    p0 = np.empty(ntraj)
    _lib.call("rpm_singlet_population", _lib.ptr(psi), n, ntraj, ld, _lib.dptr(p0), _lib.stream_handle())
    values[:, 0] = p0
    errors[:, 0] = 0.0
    accumulated = np.zeros(ntraj)
    accepted = np.zeros(ntraj, dtype=np.int64)
    matvecs = np.zeros(ntraj, dtype=np.int64)
    min_step = np.full(ntraj, np.inf)
    max_step = np.zeros(ntraj)
    cursor, current = 1, 0.0
    for k, seg in enumerate(segs):
        boundary = float(seg.end_us)
        stop = int(np.searchsorted(times, boundary + 1e-12, side="right"))
        requested = times[cursor:stop] - current
        duration = boundary - current
        local = requested if requested.size and requested[-1] >= duration - 1e-12 else np.append(requested, duration)
        idx = np.asarray(seg.system_index, dtype=np.int32)
        bp = first if k == 0 else BatchedPropagator(seg.hamiltonians, krylov_dimension=krylov_dimension,
                                                    state_error_budget=budget_of(k), **knobs)
        if bp.leading_dimension != ld:
            raise ValueError("all segments must use systems of the same dimensions")
        vals, errs, stats = bp.propagate_device(psi, local, idx)
        count = requested.size
        v = vals[:, :count].cpu().numpy()
        e = errs[:, :count].cpu().numpy()
        values[:, cursor:stop] = v
        errors[:, cursor:stop] = accumulated[:, None] + e
        bad = [int(s.status) for s in stats if s.status]
        if bad:
            raise RuntimeError(STATUS_TEXT.get(bad[0], f"batched propagation failed (status {bad[0]})"))
        accumulated += np.array([s.accumulated_state_error for s in stats])
        accepted += np.array([s.accepted_steps for s in stats])
        matvecs += np.array([s.matvecs for s in stats])
        min_step = np.minimum(min_step, [s.minimum_step_us if s.accepted_steps else np.inf for s in stats])
        max_step = np.maximum(max_step, [s.maximum_step_us for s in stats])
        cursor, current = stop, boundary
        if seg.pulse is not None and boundary < times[-1] - 1e-12:
            axis, unitary = seg.pulse
            op = np.ascontiguousarray(unitary, dtype=np.complex128)
            dd = np.ascontiguousarray(dims, dtype=np.int32)
            out = torch.empty_like(psi)
            _lib.call("rpm_apply_local_operator", _lib.iptr(dd), len(dd), int(axis), op.ctypes.data_as(_lib._PD),
                      _lib.ptr(psi), _lib.ptr(out), ntraj, ld, _lib.stream_handle())
            psi = out
    yields = None
    if lifetime_us is not None:
        vt = torch.from_numpy(np.ascontiguousarray(values)).to("cuda")
        t = torch.as_tensor(times, device="cuda")
        out = torch.empty(ntraj, dtype=torch.float64, device="cuda")
        _lib.call("rpm_simpson_yield", _lib.ptr(t), _lib.ptr(vt), int(times.size), ntraj, int(times.size),
                  float(lifetime_us), _lib.ptr(out), _lib.stream_handle())
        yields = out.cpu().numpy()
    bounds = population_bounds(errors)
    st = tuple(PropagationStats(int(accepted[b]), 0, int(matvecs[b]), int(krylov_dimension),
                                float(min_step[b]) if np.isfinite(min_step[b]) else 0.0, float(max_step[b]),
                                float(accumulated[b]), 0.0) for b in range(ntraj))
    return BatchedResult(times, values, bounds, errors, yields, psi, st, np.zeros(ntraj, dtype=np.int32))


class ConcurrentBatches:
    """Trajectories split into ``parts`` independent batches that run on their
    own streams at the same time (one host thread per part).

    Each part is a :class:`BatchedPropagator` whose persistent Lanczos launches
    leave ``reserve_sms`` SMs free, so that while one part runs its Lanczos
    iterations the other's controller, Gram, rebuild and observation kernels
    run on the free SMs instead of waiting.  Results are those of the parts
    (same arithmetic per trajectory) in the caller's order.
    """

    def __init__(self, hamiltonians: Sequence[MatrixFreeHamiltonian], *, parts: int = 2, reserve_sms: int = 16,
                 **knobs) -> None:
        torch = _torch()
        if parts < 1:
            raise ValueError("parts must be positive")
        sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
        ctas = max(1, sms - int(reserve_sms)) if parts > 1 else 0
        self.parts = [BatchedPropagator(hamiltonians, persistent_ctas=ctas, **knobs) for _ in range(parts)]
        self.streams = [torch.cuda.Stream() for _ in range(parts)]
        self.hamiltonians = self.parts[0].hamiltonians
        self.leading_dimension = self.parts[0].leading_dimension

    def _spans(self, n: int):
        k = len(self.parts)
        edges = [round(i * n / k) for i in range(k + 1)]
        return [(edges[i], edges[i + 1]) for i in range(k) if edges[i + 1] > edges[i]]

    def propagate_device(self, psi, times_us, system_index):
        """As :meth:`BatchedPropagator.propagate_device` on a (trajectories, ld)
        buffer; the parts take contiguous row blocks."""
        import threading

        torch = _torch()
        idx = np.ascontiguousarray(system_index, dtype=np.int32)
        spans = self._spans(idx.size)
        out = [None] * len(spans)
        errors = []
        caller = torch.cuda.current_stream()

        def run(k, a, b):
            try:
                s = self.streams[k]
                s.wait_stream(caller)
                with torch.cuda.stream(s):
                    out[k] = self.parts[k].propagate_device(psi[a:b], times_us, idx[a:b], stream=s)
            except Exception as exc:  # re-raised in the caller
                errors.append(exc)

        threads = [threading.Thread(target=run, args=(k, a, b)) for k, (a, b) in enumerate(spans)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if errors:
            raise errors[0]
        for s in self.streams[: len(spans)]:
            caller.wait_stream(s)
        values = torch.cat([o[0] for o in out])
        errs = torch.cat([o[1] for o in out])
        stats = [st for o in out for st in o[2]]
        return values, errs, stats

    def counters(self, reset: bool = False) -> dict:
        got = [p.counters(reset) for p in self.parts]
        n = sum(g["hpsi_samples"] for g in got)
        return {"kernel_launches": sum(g["kernel_launches"] for g in got),
                "step_replays": sum(g["step_replays"] for g in got),
                "hpsi_ms": sum(g["hpsi_ms"] * g["hpsi_samples"] for g in got) / n if n else 0.0,
                "hpsi_samples": n}

    def lanczos_kind(self) -> str:
        return self.parts[0].lanczos_kind()

    def yields_device(self, times_us, values, lifetime_us: float):
        return self.parts[0].yields_device(times_us, values, lifetime_us)

    def propagate(self, initial_states, times_us, *, system_index=None, lifetime_us=None):
        """The public path from host states: per part :meth:`BatchedPropagator.propagate`
        (host to device copies included), concurrently, results concatenated."""
        import threading

        n = len(initial_states)
        idx = np.zeros(n, dtype=np.int32) if system_index is None else np.asarray(system_index, dtype=np.int32)
        spans = self._spans(n)
        out = [None] * len(spans)
        errors = []

        def run(k, a, b):
            try:
                torch = _torch()
                with torch.cuda.stream(self.streams[k]):
                    out[k] = self.parts[k].propagate(initial_states[a:b], times_us, system_index=idx[a:b],
                                                     lifetime_us=lifetime_us)
                self.streams[k].synchronize()
            except Exception as exc:
                errors.append(exc)

        threads = [threading.Thread(target=run, args=(k, a, b)) for k, (a, b) in enumerate(spans)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if errors:
            raise errors[0]
        cat = np.concatenate
        return BatchedResult(out[0].times_us, cat([o.observable_values for o in out]),
                             cat([o.observable_error_bounds for o in out]),
                             cat([o.state_error_estimates for o in out]),
                             None if out[0].yields is None else cat([o.yields for o in out]), None,
                             tuple(s for o in out for s in o.stats), cat([o.status for o in out]))
