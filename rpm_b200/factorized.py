"""Factorized exact ensemble singlet yields on the GPU (rpm_quantum_needle_reproduction.py:93-240).

For an uncoupled radical pair (no exchange or dipolar term, D = J = 0) the
Hamiltonian is H_A (x) 1 + 1 (x) H_B and the random-phase ensemble singlet
yield with Haberkorn rate k = 1/tau factorizes:

    Phi_S(tau) = 1/4 + sum_{p,q in x,y,z} sum_{lines a of A, b of B}
                 c^A_pq(a) c^B_pq(b) k / (k - i (w_a + w_b)),

a line of a radical being a pair of its eigenstates (i, j) with frequency
w = lambda_i - lambda_j and weight <i|S_p|j><j|S_q|i> / (nuclear dimension).
As in the reference, the lines of each radical are binned with linear
interpolation onto a frequency grid of spacing (1 / tau_max) / bins, the
two spectra are convolved by FFT, and the kernel k / (k - i w) is summed over
the convolved grid.

GPU work: the radical blocks come from the library's split tables; their
eigen-decompositions use the GPU batched Hermitian eigen-solver, the spin
operators are rotated into the eigenbases with GPU matrix products, the
lines are binned by the library's ``rpm_bin_transition_lines`` kernel
(FP64), and the convolution is a GPU FFT.
"""

from __future__ import annotations

import math
from typing import Iterable, Sequence

import numpy as np

from . import _lib
from .engine import _torch

_SPIN_HALF = (np.array([[0.0, 0.5], [0.5, 0.0]], dtype=complex),
              np.array([[0.0, -0.5j], [0.5j, 0.0]], dtype=complex),
              np.array([[0.5, 0.0], [0.0, -0.5]], dtype=complex))


def _next_fast_len(n: int) -> int:
    """Smallest 2^a 3^b 5^c 7^d >= n (an efficient FFT length)."""
    best = 1 << (int(n - 1).bit_length())
    p7 = 1
    while p7 < best:
        p5 = p7
        while p5 < best:
            p3 = p5
            while p3 < best:
                p2 = p3
                while p2 < n:
                    p2 *= 2
                best = min(best, p2)
                p3 *= 3
            p5 *= 5
        p7 *= 7
    return best


def radical_blocks(hamiltonian) -> tuple[np.ndarray, np.ndarray]:
    """Dense radical operators (electron digit slowest) of an uncoupled pair."""
    pair = np.asarray(hamiltonian.electron_pair_operator).reshape(4, 4)
    if np.max(np.abs(pair)) != 0.0:
        raise ValueError("The factorized yield needs an uncoupled radical pair (no electron-pair term).")
    return hamiltonian.left_operator.toarray(), hamiltonian.right_operator.toarray()


class _Spectrum:
    def __init__(self, torch, block: np.ndarray):
        h = torch.from_numpy(np.ascontiguousarray(block)).to("cuda")
        h = 0.5 * (h + h.conj().T)
        self.lam, vec = torch.linalg.eigh(h)
        d = block.shape[0]
        self.d = d
        self.nuclear = d // 2
        v3 = vec.reshape(2, self.nuclear, d)
        self.ops = []
        for s in _SPIN_HALF:
            st = torch.from_numpy(s).to("cuda")
            w = torch.einsum("ef,fnk->enk", st, v3).reshape(d, d)
            self.ops.append((vec.conj().T @ w).contiguous())
        self.max_gap = float((self.lam.max() - self.lam.min()).item())


def _binned(torch, spec: _Spectrum, p: int, q: int, delta: float, half: int, bad):
    grid = torch.zeros(2 * half + 1, dtype=torch.complex128, device="cuda")
    _lib.call("rpm_bin_transition_lines", _lib.ptr(spec.lam), _lib.ptr(spec.ops[p]), _lib.ptr(spec.ops[q]), spec.d,
              1.0 / spec.nuclear, float(delta), int(half), _lib.ptr(grid), _lib.ptr(bad), _lib.stream_handle())
    return grid


def factorized_singlet_yields(hamiltonians: Sequence, lifetimes_us: Iterable[float], *,
                              bins_per_linewidth: float = 8.0) -> tuple[np.ndarray, np.ndarray]:
    """Ensemble singlet yields (n_hamiltonians, n_lifetimes) and initial singlet populations.

    ``hamiltonians``: uncoupled :class:`CompiledFullPairHamiltonian` objects
    (e.g. one per field orientation).  Mirrors ``solve_orientation`` and
    ``convolved_correlation_spectrum`` of the reference
    (rpm_quantum_needle_reproduction.py:172-240).
    """
    torch = _torch()
    lifetimes = tuple(float(t) for t in lifetimes_us)
    if not lifetimes or min(lifetimes) <= 0.0:
        raise ValueError("Lifetimes must be positive.")
    if bins_per_linewidth < 2.0:
        raise ValueError("bins_per_linewidth must be at least 2.")
    delta = (1.0 / max(lifetimes)) / float(bins_per_linewidth)
    yields = np.empty((len(hamiltonians), len(lifetimes)))
    initial = np.empty(len(hamiltonians))
    bad = torch.zeros(1, dtype=torch.int32, device="cuda")
    for row, h in enumerate(hamiltonians):
        blk_a, blk_b = radical_blocks(h)
        spec_a, spec_b = _Spectrum(torch, blk_a), _Spectrum(torch, blk_b)
        margin = 3
        half_a = int(math.ceil(spec_a.max_gap / delta)) + margin
        half_b = int(math.ceil(spec_b.max_gap / delta)) + margin
        out_len = (2 * half_a + 1) + (2 * half_b + 1) - 1
        nfft = _next_fast_len(out_len)
        combined = torch.zeros(nfft, dtype=torch.complex128, device="cuda")
        for p in range(3):
            for q in range(3):
                ga = _binned(torch, spec_a, p, q, delta, half_a, bad)
                gb = _binned(torch, spec_b, p, q, delta, half_b, bad)
                combined += torch.fft.fft(ga, n=nfft) * torch.fft.fft(gb, n=nfft)
        if int(bad.item()):
            raise ValueError("Frequency grid is too small for transition spectrum.")
        conv = torch.fft.ifft(combined)[:out_len]
        omega = (torch.arange(out_len, dtype=torch.float64, device="cuda") - (half_a + half_b)) * delta
        initial[row] = float((0.25 + conv.sum()).real.item())
        for col, tau in enumerate(lifetimes):
            k = 1.0 / tau
            kern = k / (k - 1j * omega)
            yields[row, col] = float((0.25 + (conv * kern).sum()).real.item())
    return yields, initial
