"""Segment propagation: instantaneous local unitaries and piecewise-constant fields.

Mirrors the reference's pulsed-control loop
(``rpm_nuclear_spin_rotation_control.py:281-308``): the horizon is cut at the
pulse times; every segment is propagated by a fresh
``AdaptiveLanczosPropagator`` whose state-error budget is the total budget
scaled by the segment's duration; observation points inside a segment are
reported with the errors accumulated by earlier segments; between segments a
d x d unitary is applied to one tensor axis (``core.py:285-292``, on the GPU).
A segment may also carry its own Hamiltonian, which turns the same loop into a
propagator for piecewise-constant fields (a square field pulse is three
segments).
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _lib
from .engine import AdaptiveLanczosPropagator, SingletPopulationObservable, _as_device, _torch, singlet_population
from .model import spin_operators


def local_unitary_apply(state, dimensions: Sequence[int], axis: int, unitary):
    """Apply a d x d operator to one tensor axis on the GPU (core.py:285-292)."""
    torch = _torch()
    dims = np.ascontiguousarray(dimensions, dtype=np.int32)
    n = int(np.prod(dims))
    flat = state.reshape(-1) if isinstance(state, torch.Tensor) else np.asarray(state, dtype=complex).reshape(-1)
    x, host = _as_device(flat, n, torch)
    d = int(dims[axis])
    op = np.ascontiguousarray(unitary, dtype=np.complex128)
    if op.shape != (d, d):
        raise ValueError(f"operator shape {op.shape} does not match axis dimension {d}")
    out = torch.empty_like(x)
    _lib.call("rpm_apply_local_operator", _lib.iptr(dims), len(dims), int(axis), op.ctypes.data_as(_lib._PD),
              _lib.ptr(x), _lib.ptr(out), 1, n, _lib.stream_handle())
    return out.cpu().numpy() if host else out


def spin_pi_pulse(spin: float, molecular_axis) -> np.ndarray:
    """exp(-i pi n.S) for a unit axis n (core.py:304-308), built on the host."""
    n = np.asarray(molecular_axis, dtype=float)
    n = n / np.linalg.norm(n)
    gen = sum(c * op for c, op in zip(n, spin_operators(spin)))
    w, v = np.linalg.eigh(gen)
    return (v * np.exp(-1j * math.pi * w)) @ v.conj().T


@dataclass(frozen=True)
class Segment:
    """Propagate with ``hamiltonian`` until ``end_us``, then apply ``pulse``
    (``(axis, unitary)`` or None) unless ``end_us`` is the final time."""

    end_us: float
    hamiltonian: object
    pulse: tuple | None = None


@dataclass(frozen=True)
class SegmentResult:
    times_us: np.ndarray
    observable_values: np.ndarray
    observable_error_bounds: np.ndarray
    state_error_estimates: np.ndarray
    final_state: np.ndarray
    accepted_steps: int
    rejected_steps: int
    matvecs: int
    accumulated_state_error: float


def propagate_segments(initial_state, times_us, segments: Sequence[Segment], *, state_error_budget: float = 2.4e-5,
                       **knobs) -> SegmentResult:
    """Singlet populations through a sequence of segments (see module docstring).

    ``times_us`` must start at 0; the last segment must end at its last time.
    ``knobs`` are passed to every segment's AdaptiveLanczosPropagator.
    """
    times = np.asarray(times_us, dtype=float)
    if times.ndim != 1 or times.size == 0 or times[0] != 0.0 or np.any(np.diff(times) <= 0.0):
        raise ValueError("Observation times must start at 0 and be strictly increasing.")
    segs = list(segments)
    if not segs or not math.isclose(segs[-1].end_us, times[-1], rel_tol=0.0, abs_tol=1e-12):
        raise ValueError("The last segment must end at the final observation time.")
    ends = [s.end_us for s in segs]
    if any(b <= a for a, b in zip(ends, ends[1:])) or ends[0] <= 0.0:
        raise ValueError("Segment end times must be positive and strictly increasing.")
    dims = segs[0].hamiltonian.dimensions
    observable = SingletPopulationObservable(dims)
    state = np.asarray(initial_state, dtype=complex).reshape(-1)
    values = np.empty(times.size)
    bounds = np.empty(times.size)
    errors = np.empty(times.size)
    values[0] = singlet_population(state, dims)
    bounds[0] = errors[0] = 0.0
    cursor, current = 1, 0.0
    accepted = rejected = matvecs = 0
    accumulated = 0.0
    for seg in segs:
        boundary = float(seg.end_us)
        stop = int(np.searchsorted(times, boundary + 1e-12, side="right"))
        requested = times[cursor:stop] - current
        duration = boundary - current
        if requested.size == 0 or requested[-1] < duration - 1e-12:
            local = np.append(requested, duration)
        else:
            local = requested
        if duration > 0.0:
            prop = AdaptiveLanczosPropagator(seg.hamiltonian, **knobs)
            prop.state_error_budget = state_error_budget * duration / times[-1]
            res = prop.propagate(state, local, observable)
            count = requested.size
            values[cursor:stop] = res.observable_values[:count]
            glob = accumulated + res.state_error_estimates[:count]
            errors[cursor:stop] = glob
            bounds[cursor:stop] = 2.0 * glob + glob ** 2
            state = res.final_state
            accepted += res.stats.accepted_steps
            rejected += res.stats.rejected_steps
            matvecs += res.stats.matvecs
            accumulated += res.stats.accumulated_state_error
        cursor = stop
        current = boundary
        if seg.pulse is not None and boundary < times[-1] - 1e-12:
            axis, unitary = seg.pulse
            state = local_unitary_apply(state, dims, axis, unitary)
    return SegmentResult(times, values, bounds, errors, np.asarray(state), accepted, rejected, matvecs, accumulated)


def square_pulse_segments(h_static, h_pulse, start_us: float, duration_us: float, end_us: float) -> list[Segment]:
    """Static field, then the pulsed field on [start, start + duration), then static again."""
    out = []
    if start_us > 0.0:
        out.append(Segment(start_us, h_static))
    out.append(Segment(start_us + duration_us, h_pulse))
    if start_us + duration_us < end_us:
        out.append(Segment(end_us, h_static))
    return out
