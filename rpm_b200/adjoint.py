"""Gradients of the singlet yield by an adjoint sweep on the GPU.

No reference implementation exists: the reference differentiates yields only
by finite differences over angle grids (``np.gradient`` over theta in
``rpm_quantum_needle_reproduction.py`` and ``rpm_three_nitrogen_quadrupole.py``).
Here the yield of a trajectory on a uniform observation grid,

    Phi = sum_k w_k <psi_k| P_S |psi_k>,   w_k = Simpson weight * exp(-t_k/tau) / tau,

is differentiated with respect to the parameters of
:class:`ParametricRadicalPair` -- static field magnitude and direction
(|B|, theta, phi), the amplitude of a transverse square field pulse and a
global hyperfine scale -- through

    dPhi/dp = sum_k 2 Im int_{t_k}^{t_k+1} <lambda(t)| dH/dp |psi(t)> dt,

with the adjoint lambda_k = U_k^dag lambda_{k+1} + w_k P_S psi_k marched
backwards over the grid (``rpm_adjoint_sweep``, ``csrc/adjoint.cu``).

Checkpoints: the forward pass runs block by block and keeps each block's end
state (complex128).  The backward pass restarts psi from the checkpoint at
the end of each block (last block first) and recomputes it interval by
interval backwards together with lambda (equal-rate evolution is unitary, so
the backward recomputation is as stable as the forward one); the drift
between the recomputed psi at the block start and the checkpoint there is
reported.

Precision.  The gradient's sensitivity to errors of the states grows with
||dH/dp|| times the horizon.  Field derivatives (Zeeman-sized operators) are
well conditioned and the complex64 path -- forward by the batched
mixed-precision Krylov propagator with blocks of about ``checkpoint_steps``
Krylov steps, backward with a complex64 Taylor basis -- meets 1e-4.  The
hyperfine part is most of H: its derivative needs states accurate to about
1e-9, which complex64 arithmetic does not give, so ``precision="c128"``
runs both passes with the complex128 Taylor basis (fixed schedule, blocks of
``checkpoint_intervals`` grid intervals).

Field derivatives are electron-pair operators, contracted with the
accumulated transition densities.  For the hyperfine scale s,
dH/ds = (H - Zeeman - exchange/dipolar - quadrupole) / s: <lambda| H |psi> is
constant over each interval and taken once per interval in FP64, the
electron terms come from the transition densities and the (small)
quadrupole part from a quadrupole-only system at the quadrature nodes.

:func:`singlet_yield` wraps forward and backward as a
``torch.autograd.Function`` of the parameter tensor.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .batched import STATUS_TEXT, BatchedPropagator
from .engine import CompiledFullPairHamiltonian, _torch
from .model import zeeman_operator

PARAMETERS = ("field_microT", "theta", "phi", "pulse_nT", "hyperfine_scale")
TAYLOR_TOLERANCE = 1e-10
PRECISIONS = {"c64": _lib.PREC_C64, "c128": _lib.PREC_C128}


def simpson_weights(times_us) -> np.ndarray:
    """Weights c_k with Simpson(y, t) = sum_k c_k y_k, for the composite rule of
    ``rpm_simpson_yield`` (scipy.integrate.simpson; odd counts: classic panels,
    even counts: the last interval by the three-point end correction)."""
    t = np.asarray(times_us, dtype=float)
    n = t.size
    c = np.zeros(n)
    if n == 1:
        return c
    if n == 2:
        c[:] = 0.5 * (t[1] - t[0])
        return c
    stop = n - 1 if n % 2 == 1 else n - 2
    k = np.arange(0, stop - 1, 2)
    h0 = t[k + 1] - t[k]
    h1 = t[k + 2] - t[k + 1]
    hs, hp, r = h0 + h1, h0 * h1, h0 / h1
    np.add.at(c, k, hs / 6.0 * (2.0 - 1.0 / r))
    np.add.at(c, k + 1, hs / 6.0 * (hs * hs / hp))
    np.add.at(c, k + 2, hs / 6.0 * (2.0 - r))
    if n % 2 == 0:
        a, b = t[n - 2] - t[n - 3], t[n - 1] - t[n - 2]
        c[n - 1] += (2 * b * b + 3 * a * b) / (6 * (a + b))
        c[n - 2] += (b * b + 3 * a * b) / (6 * a)
        c[n - 3] -= b * b * b / (6 * a * (a + b))
    return c


def yield_weights(times_us, lifetime_us: float) -> np.ndarray:
    """w_k of Phi = sum_k w_k P_S(t_k): Simpson weights times exp(-t/tau)/tau."""
    t = np.asarray(times_us, dtype=float)
    return simpson_weights(t) * np.exp(-t / lifetime_us) / lifetime_us


def electron_pair_zeeman(field_mT) -> np.ndarray:
    """4 x 4 operator Z(B) (x) 1 + 1 (x) Z(B) on (eA, eB), index 2 eA + eB."""
    z = zeeman_operator(np.asarray(field_mT, dtype=float))
    eye = np.eye(2)
    return np.kron(z, eye) + np.kron(eye, z)


def _unit_vectors(theta: float, phi: float):
    st, ct, sp, cp = math.sin(theta), math.cos(theta), math.sin(phi), math.cos(phi)
    n = np.array([st * cp, st * sp, ct])
    e_theta = np.array([ct * cp, ct * sp, -st])
    e_phi = np.array([-sp, cp, 0.0])
    return n, e_theta, e_phi


class ParametricRadicalPair:
    """H(p, t) of a :class:`rpm_b200.synthetic.SyntheticSystem` with parameters
    p = (|B| in uT, theta, phi in rad, pulse amplitude in nT, hyperfine scale):

        B(t) = |B| n(theta, phi) + a [t in pulse] e_theta(theta, phi)

    (the pulse is transverse to the static field, along the polar unit
    vector), electron Zeeman on both electrons, hyperfine terms times the
    scale, quadrupole and exchange/dipolar terms fixed."""

    def __init__(self, system, *, pulse_start_us: float = 0.2, pulse_duration_us: float = 0.5) -> None:
        self.system = system
        self.pulse_start_us = float(pulse_start_us)
        self.pulse_duration_us = float(pulse_duration_us)
        self._quadrupole = None

    @property
    def dimensions(self):
        return self.system.dimensions

    def _hamiltonian(self, terms) -> CompiledFullPairHamiltonian:
        s = self.system
        return CompiledFullPairHamiltonian(s.dimensions, terms, left_axes=s.left_axes, right_axes=s.right_axes)

    def pulse_field_mT(self, params) -> np.ndarray:
        _, e_theta, _ = _unit_vectors(float(params[1]), float(params[2]))
        return 1e-6 * float(params[3]) * e_theta

    def field_mT(self, params) -> np.ndarray:
        """Field of each segment [static, pulsed], mT, shape (2, 3)."""
        n, _, _ = _unit_vectors(float(params[1]), float(params[2]))
        static = 1e-3 * float(params[0]) * n
        return np.stack([static, static + self.pulse_field_mT(params)])

    def hamiltonians(self, params):
        """(static, pulsed) Hamiltonians at ``params``."""
        b, th, ph, _, scale = (float(v) for v in params)
        static = self.system.terms(th, ph, field_microT=b, hyperfine_scale=scale)
        pulsed = self.system.terms(th, ph, field_microT=b, hyperfine_scale=scale,
                                   extra_field_mT=self.pulse_field_mT(params))
        return self._hamiltonian(static), self._hamiltonian(pulsed)

    def quadrupole_system(self):
        """The nuclear quadrupole terms alone (None when the system has none)."""
        if self._quadrupole is None:
            terms = [t for t in self.system.terms(0.0, 0.0, field_microT=0.0) if t.label.endswith("quadrupole")]
            self._quadrupole = self._hamiltonian(terms) if terms else False
        return self._quadrupole or None

    def electron_pair_operator(self) -> np.ndarray:
        """The fixed exchange + dipolar operator on (eA, eB), 4 x 4 (zero if absent)."""
        for t in self.system.terms(0.0, 0.0, field_microT=0.0):
            if tuple(t.axes) == (0, 1):
                return np.asarray(t.operator, dtype=complex)
        return np.zeros((4, 4), dtype=complex)

    def field_derivatives_mT(self, params) -> np.ndarray:
        """dB/dp (mT per unit of p), shape (2 segments [static, pulsed], 5 parameters, 3)."""
        b, th, _, a, _ = (float(v) for v in params)
        n, e_theta, e_phi = _unit_vectors(th, float(params[2]))
        d = np.zeros((2, 5, 3))
        for seg in (0, 1):
            pulse = 1e-6 * a if seg == 1 else 0.0
            d[seg, 0] = 1e-3 * n
            d[seg, 1] = 1e-3 * b * e_theta - pulse * n
            d[seg, 2] = 1e-3 * b * math.sin(th) * e_phi + pulse * math.cos(th) * e_phi
            d[seg, 3] = 1e-6 * e_theta if seg == 1 else 0.0
        return d

    def electron_derivatives(self, params) -> np.ndarray:
        """Electron-pair parts of dH/dp for the field parameters, shape (2, 5, 4, 4)."""
        d = self.field_derivatives_mT(params)
        out = np.zeros((2, 5, 4, 4), dtype=complex)
        for seg in (0, 1):
            for p in range(4):
                out[seg, p] = electron_pair_zeeman(d[seg, p])
        return out

    def interval_segments(self, times_us) -> np.ndarray:
        """Segment of each observation interval: 1 inside the pulse, else 0.
        The pulse edges must fall on grid points (or outside the grid)."""
        t = np.asarray(times_us, dtype=float)
        dt = t[1] - t[0]
        start, end = self.pulse_start_us, self.pulse_start_us + self.pulse_duration_us
        for edge in (start, end):
            if t[0] < edge < t[-1] and abs((edge - t[0]) / dt - round((edge - t[0]) / dt)) > 1e-6:
                raise ValueError("the pulse edges must fall on observation times")
        mid = 0.5 * (t[:-1] + t[1:])
        return ((mid > start) & (mid < end)).astype(np.int32)


@dataclass
class GradientResult:
    yields: np.ndarray            # (trajectories,)
    gradients: np.ndarray         # (trajectories, 5) dPhi/dp in PARAMETERS order
    populations: np.ndarray       # (trajectories, times)
    diagnostics: dict = field(default_factory=dict)


def _uniform_grid(times_us) -> tuple[np.ndarray, float]:
    t = np.asarray(times_us, dtype=float)
    if t.ndim != 1 or t.size < 2 or t[0] != 0.0:
        raise ValueError("observation times must start at 0 and hold at least two points")
    dt = float(t[1] - t[0])
    if not dt > 0.0 or np.max(np.abs(np.diff(t) - dt)) > 1e-9 * max(1.0, t[-1]):
        raise ValueError("the adjoint sweep needs a uniform observation grid")
    return t, dt


def spectral_radius(hamiltonian, *, iterations: int = 40, seed: int = 7) -> float:
    """Largest |Ritz value| of an FP64 Lanczos basis grown from a random vector
    (``rpm_lanczos_basis``): a close lower estimate of ||H||."""
    torch = _torch()
    n = hamiltonian.dimension
    m = int(min(iterations, n))
    rng = np.random.default_rng(seed)
    v = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    state = torch.as_tensor(v / np.linalg.norm(v), dtype=torch.complex128, device="cuda")
    basis = torch.empty((m, n), dtype=torch.complex128, device="cuda")
    alpha = torch.zeros(m, dtype=torch.float64, device="cuda")
    beta = torch.zeros(max(m - 1, 1), dtype=torch.float64, device="cuda")
    actual, norm = ctypes.c_int(0), ctypes.c_double(0.0)
    _lib.call("rpm_lanczos_basis", hamiltonian._system.handle, _lib.ptr(state), m, 1e-14, _lib.ptr(basis),
              _lib.ptr(alpha), _lib.ptr(beta), ctypes.byref(actual), ctypes.byref(norm), _lib.stream_handle())
    k = actual.value
    a = alpha[:k].cpu().numpy()
    b = beta[:max(k - 1, 0)].cpu().numpy()
    t = np.diag(a) + np.diag(b, 1) + np.diag(b, -1)
    return float(np.max(np.abs(np.linalg.eigvalsh(t))))


def taylor_degree(radius_dt: float, tolerance: float = TAYLOR_TOLERANCE) -> int:
    """Smallest d with (rho dt)^(d+1) / (d+1)! <= tolerance."""
    term, d = radius_dt, 0
    while term > tolerance:
        d += 1
        term *= radius_dt / (d + 1)
        if d > 24:
            raise ValueError("observation interval too long for the Taylor sweep (rho dt too large)")
    return max(d, 1)


class _Workspace:
    """Owner of an ``rpm_adjoint*`` handle."""

    def __init__(self, ntraj: int, n: int, ld: int, degree: int, nodes: int, precision: int) -> None:
        self.handle = ctypes.c_void_p()
        _lib.call("rpm_adjoint_create", int(ntraj), int(n), int(ld), int(degree), int(nodes), int(precision),
                  ctypes.byref(self.handle))
        self.degree = degree

    def close(self) -> None:
        if self.handle is not None and self.handle.value:
            _lib.call("rpm_adjoint_destroy", self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _system_array(*hams):
    return (ctypes.c_void_p * len(hams))(*(h._system.handle if h is not None else None for h in hams))


class AdjointYieldGradient:
    """Yields and their parameter gradients for many trajectories of one
    :class:`ParametricRadicalPair` on a uniform grid (equal recombination
    rates, lifetime ``lifetime_us``).  ``precision``: "c64" (complex64 Krylov
    forward and Taylor basis) or "c128" (complex128 Taylor basis in both
    passes; needed for the hyperfine-scale derivative at 1e-4)."""

    def __init__(self, model: ParametricRadicalPair, *, precision: str = "c128", krylov_dimension: int = 32,
                 state_error_budget: float = 5e-7, checkpoint_steps: int = 16, checkpoint_intervals: int = 256,
                 quadrature_nodes: int = 3, taylor_tolerance: float = TAYLOR_TOLERANCE,
                 first_block_intervals: int = 64) -> None:
        if precision not in PRECISIONS:
            raise ValueError("precision must be 'c64' or 'c128'")
        self.model = model
        self.precision = precision
        self.krylov_dimension = int(krylov_dimension)
        self.state_error_budget = float(state_error_budget)
        self.checkpoint_steps = int(checkpoint_steps)
        self.checkpoint_intervals = int(checkpoint_intervals)
        self.quadrature_nodes = int(quadrature_nodes)
        self.taylor_tolerance = float(taylor_tolerance)
        self.first_block_intervals = int(first_block_intervals)
        if self.checkpoint_steps < 1 or self.checkpoint_intervals < 1 or not 1 <= self.quadrature_nodes <= 4:
            raise ValueError("checkpoint spacing >= 1 and quadrature_nodes in 1..4 are required")

    # forward ------------------------------------------------------------
    def forward(self, params, initial_states, times_us, lifetime_us: float):
        """Yields, populations and the checkpoints of the forward pass."""
        torch = _torch()
        t, dt = _uniform_grid(times_us)
        params = np.asarray(params, dtype=float)
        h_static, h_pulse = self.model.hamiltonians(params)
        hams = (h_static, h_pulse)
        seg = self.model.interval_segments(t)
        ntraj = len(initial_states)
        radius = 1.1 * max(spectral_radius(h_static), spectral_radius(h_pulse))
        degree = taylor_degree(radius * dt, self.taylor_tolerance)
        n = int(np.prod(self.model.dimensions))
        # the batched propagator fixes the state layout (leading dimension)
        idx = np.zeros(ntraj, dtype=np.int32)
        rate = self.state_error_budget / t[-1]
        props = {}

        def propagator(kind: int, intervals: int) -> BatchedPropagator:
            if kind not in props:
                props[kind] = BatchedPropagator([hams[kind]], krylov_dimension=self.krylov_dimension,
                                                state_error_budget=rate * intervals * dt)
            props[kind].set_state_error_budget(rate * intervals * dt)
            return props[kind]

        first = propagator(int(seg[0]), 1)
        psi = first.load_states(initial_states, idx)
        ld = first.leading_dimension
        work = _Workspace(ntraj, n, ld, degree, self.quadrature_nodes, PRECISIONS[self.precision])
        pops = torch.empty((ntraj, t.size), dtype=torch.float64, device="cuda")
        p0 = np.empty(ntraj)
        _lib.call("rpm_singlet_population", _lib.ptr(psi), n, ntraj, ld, _lib.dptr(p0), _lib.stream_handle())
        pops[:, 0] = torch.as_tensor(p0, device="cuda")
        checkpoints = {0: psi.clone()}
        blocks = []
        steps_total, worst_tail = 0, 0.0
        stream = _lib.stream_handle()
        systems = _system_array(h_static, h_pulse)
        k, length = 0, (self.first_block_intervals if self.precision == "c64" else self.checkpoint_intervals)
        while k < t.size - 1:
            kind = int(seg[k])
            stop = min(k + length, t.size - 1)
            if self.precision == "c64":
                run_end = k
                while run_end < t.size - 1 and seg[run_end] == kind:
                    run_end += 1
                stop = min(stop, run_end)
                bp = propagator(kind, stop - k)
                vals, _, stats = bp.propagate_device(psi, t[k + 1:stop + 1] - t[k], idx)
                bad = [int(s.status) for s in stats if s.status]
                if bad:
                    raise RuntimeError(STATUS_TEXT.get(bad[0], f"batched propagation failed (status {bad[0]})"))
                pops[:, k + 1:stop + 1] = vals
                steps = max(int(s.accepted_steps) for s in stats)
                steps_total += steps
                if not blocks and steps > 0:
                    length = max(8, int(round(self.checkpoint_steps * (stop - k) / steps)))
            else:
                segs = np.ascontiguousarray(seg[k:stop], dtype=np.int32)
                tail = ctypes.c_double(0.0)
                out = pops[:, k + 1:]
                _lib.call("rpm_adjoint_forward", work.handle, systems, 2, _lib.iptr(segs), float(dt), int(stop - k),
                          _lib.ptr(psi), _lib.ptr(out), int(t.size), ctypes.byref(tail), stream)
                worst_tail = max(worst_tail, tail.value)
            blocks.append((k, stop))
            checkpoints[stop] = psi.clone()
            k = stop
        w = yield_weights(t, lifetime_us)
        yields = (pops * torch.as_tensor(w, device="cuda")).sum(dim=1)
        return {"times": t, "dt": dt, "segments": seg, "hamiltonians": hams, "populations": pops,
                "yields": yields, "weights": w, "blocks": blocks, "checkpoints": checkpoints, "ld": ld,
                "krylov_steps": steps_total, "workspace": work, "spectral_radius_bound": radius,
                "forward_taylor_tail": worst_tail}

    # backward -----------------------------------------------------------
    def backward(self, params, fwd):
        """Per-trajectory gradients (trajectories, 5) from a forward record."""
        torch = _torch()
        params = np.asarray(params, dtype=float)
        scale = float(params[4])
        if scale == 0.0:
            raise ValueError("the hyperfine-scale gradient needs a nonzero hyperfine scale")
        t, dt, seg = fwd["times"], fwd["dt"], fwd["segments"]
        h_static, h_pulse = fwd["hamiltonians"]
        work = fwd["workspace"]
        psi_end = fwd["checkpoints"][t.size - 1]
        ntraj = psi_end.shape[0]
        n = int(np.prod(self.model.dimensions))
        quad = self.model.quadrupole_system()
        nder = 1 if quad is not None else 0
        systems = _system_array(h_static, h_pulse)
        dsys = _system_array(quad, quad)
        density = torch.zeros((ntraj, 2, 16, 2), dtype=torch.float64, device="cuda")
        deriv = torch.zeros((ntraj, 2, 1, 2), dtype=torch.float64, device="cuda")
        energy = torch.zeros((ntraj, 2, 2), dtype=torch.float64, device="cuda")
        w = fwd["weights"]
        lam = torch.zeros_like(psi_end)
        psi = psi_end.clone()
        stream = _lib.stream_handle()
        _lib.call("rpm_adjoint_source", work.handle, _lib.ptr(psi), _lib.ptr(lam), float(w[-1]), stream)
        worst_tail, drift = 0.0, 0.0
        for k0, k1 in reversed(fwd["blocks"]):
            psi.copy_(fwd["checkpoints"][k1])
            segs = np.ascontiguousarray(seg[k0:k1], dtype=np.int32)
            ws = np.ascontiguousarray(w[k0:k1], dtype=np.float64)
            tail = ctypes.c_double(0.0)
            _lib.call("rpm_adjoint_sweep", work.handle, systems, 2, dsys, nder, _lib.iptr(segs), _lib.dptr(ws),
                      float(dt), int(k1 - k0), _lib.ptr(lam), _lib.ptr(psi), _lib.ptr(density), _lib.ptr(deriv),
                      _lib.ptr(energy), ctypes.byref(tail), stream)
            worst_tail = max(worst_tail, tail.value)
            ref = fwd["checkpoints"][k0]
            drift = max(drift, float(torch.max(torch.linalg.vector_norm(psi[:, :n] - ref[:, :n], dim=1))))
        m = torch.view_as_complex(density).cpu().numpy()         # (ntraj, 2, 16)
        q = torch.view_as_complex(deriv).cpu().numpy()[:, :, 0]  # (ntraj, 2)
        en = torch.view_as_complex(energy).cpu().numpy()         # (ntraj, 2)
        e = self.model.electron_derivatives(params).reshape(2, 5, 16)
        grads = 2.0 * np.imag(np.einsum("spk,bsk->bp", e, m))
        fields = self.model.field_mT(params)
        pair = self.model.electron_pair_operator()
        rest = np.stack([electron_pair_zeeman(fields[s]) + pair for s in (0, 1)]).reshape(2, 16)
        hyperfine = en - np.einsum("sk,bsk->bs", rest, m) - q
        grads[:, 4] = 2.0 * np.imag(hyperfine.sum(axis=1)) / scale
        diag = {"precision": self.precision, "taylor_degree": work.degree,
                "spectral_radius_bound": fwd["spectral_radius_bound"],
                "max_taylor_tail": max(worst_tail, fwd["forward_taylor_tail"]), "checkpoint_drift": drift,
                "blocks": len(fwd["blocks"]), "krylov_steps": fwd["krylov_steps"]}
        return grads, diag

    def yields(self, params, initial_states, times_us, lifetime_us: float) -> np.ndarray:
        """Forward pass only (for example for finite differences through the
        same fixed-schedule path)."""
        fwd = self.forward(params, initial_states, times_us, lifetime_us)
        fwd["workspace"].close()
        return fwd["yields"].cpu().numpy()

    def __call__(self, params, initial_states, times_us, lifetime_us: float) -> GradientResult:
        fwd = self.forward(params, initial_states, times_us, lifetime_us)
        try:
            grads, diag = self.backward(params, fwd)
        finally:
            fwd["workspace"].close()
        return GradientResult(fwd["yields"].cpu().numpy(), grads, fwd["populations"].cpu().numpy(), diag)


def _autograd_function():
    torch = _torch()

    class SingletYield(torch.autograd.Function):
        """yields = SingletYield.apply(params, engine, states, times_us, lifetime_us)

        ``params``: float64 tensor of the five :data:`PARAMETERS`; returns the
        float64 yields of the trajectories.  The backward pass is the adjoint
        sweep; the gradient of a weighted sum of yields is the per-trajectory
        gradients contracted with the incoming weights."""

        @staticmethod
        def forward(ctx, params, engine, states, times_us, lifetime_us):
            p = params.detach().cpu().numpy().astype(float)
            fwd = engine.forward(p, states, times_us, lifetime_us)
            ctx.engine, ctx.fwd, ctx.p = engine, fwd, p
            return fwd["yields"].to(params.device)

        @staticmethod
        def backward(ctx, grad_yields):
            try:
                grads, _ = ctx.engine.backward(ctx.p, ctx.fwd)
            finally:
                ctx.fwd["workspace"].close()
            g = torch.as_tensor(grads, dtype=torch.float64, device=grad_yields.device)
            return grad_yields.to(torch.float64) @ g, None, None, None, None

    return SingletYield


_SINGLET_YIELD = None


def singlet_yield(params, engine: AdjointYieldGradient, initial_states, times_us, lifetime_us: float):
    """Differentiable yields: ``singlet_yield(p, engine, states, t, tau).sum().backward()``."""
    global _SINGLET_YIELD
    if _SINGLET_YIELD is None:
        _SINGLET_YIELD = _autograd_function()
    return _SINGLET_YIELD.apply(params, engine, initial_states, times_us, lifetime_us)
