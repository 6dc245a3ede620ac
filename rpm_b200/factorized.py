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

GPU work, all in the library's own FP64 kernels: the radical blocks come
from the library's split tables; their eigen-decompositions are batched over
the field orientations (``rpm_he_eigh``: Householder tridiagonalisation,
implicit tridiagonal QR, back-transformation, one CTA per matrix); the spin
operators are rotated into the eigenbases by ``rpm_zgemm_hn`` (V^H (S (x) 1)
V); the lines are binned by ``rpm_bin_transition_lines``; the two spectra
are convolved by radix-2 FFTs (``rpm_fft_pow2``, zero-padded to a power of two
no shorter than the linear convolution, which leaves the convolution itself
unchanged).
"""

from __future__ import annotations

import ctypes
import math
from typing import Iterable, Sequence

import numpy as np

from . import _lib
from .engine import _torch

_SPIN_HALF = (np.array([[0.0, 0.5], [0.5, 0.0]], dtype=complex),
              np.array([[0.0, -0.5j], [0.5j, 0.0]], dtype=complex),
              np.array([[0.5, 0.0], [0.0, -0.5]], dtype=complex))


def radical_blocks(hamiltonian) -> tuple[np.ndarray, np.ndarray]:
    """Dense radical operators (electron digit slowest) of an uncoupled pair."""
    pair = np.asarray(hamiltonian.electron_pair_operator).reshape(4, 4)
    if np.max(np.abs(pair)) != 0.0:
        raise ValueError("The factorized yield needs an uncoupled radical pair (no electron-pair term).")
    return hamiltonian.left_operator.toarray(), hamiltonian.right_operator.toarray()


def hermitian_eigh(blocks):
    """Eigenvalues (ascending) and eigenvectors (columns) of a batch of
    Hermitian matrices (device tensor, batch x n x n complex128), by the
    library's FP64 solver; the input is Hermitian-symmetrised first."""
    torch = _torch()
    a = (0.5 * (blocks + blocks.conj().transpose(-1, -2))).contiguous()
    batch, n = a.shape[0], a.shape[-1]
    lam = torch.empty((batch, n), dtype=torch.float64, device="cuda")
    vec = torch.empty((batch, n, n), dtype=torch.complex128, device="cuda")
    if n == 1:
        lam.copy_(a[:, 0, 0].real)
        vec.fill_(1.0)
        return lam, vec
    # chunks: at most 65535 matrices (grid limit) and about 2 GB of workspace
    chunk = int(max(1, min(65535, 2_000_000_000 // (48 * n * n + 64 * n))))
    for b0 in range(0, batch, chunk):
        nb = min(chunk, batch - b0)
        size = ctypes.c_longlong()
        _lib.call("rpm_he_eigh_workspace", n, nb, ctypes.byref(size))
        work = torch.empty(size.value, dtype=torch.uint8, device="cuda")
        _lib.call("rpm_he_eigh", n, nb, _lib.ptr(a[b0:b0 + nb]), _lib.ptr(lam[b0:b0 + nb]), _lib.ptr(vec[b0:b0 + nb]),
                  _lib.ptr(work), _lib.stream_handle())
    return lam, vec


class _Spectrum:
    """Eigenvalues of one radical block and its electron spin operators in the
    eigenbasis, <i| S_p (x) 1 |j>."""

    def __init__(self, torch, lam, vec):
        d = vec.shape[0]
        self.lam = lam
        self.d = d
        self.nuclear = d // 2
        v3 = vec.reshape(2, self.nuclear, d)
        self.ops = []
        for s in _SPIN_HALF:
            # (S (x) 1) V: rows of electron e are s[e, 0] V_0 + s[e, 1] V_1
            w = torch.cat([complex(s[e, 0]) * v3[0] + complex(s[e, 1]) * v3[1] for e in (0, 1)]).contiguous()
            op = torch.empty_like(w)
            _lib.call("rpm_zgemm_hn", d, 1, _lib.ptr(vec), _lib.ptr(w), _lib.ptr(op), _lib.stream_handle())
            self.ops.append(op)
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
    blocks = [radical_blocks(h) for h in hamiltonians]
    # one batched eigen-decomposition per radical over all orientations
    eig_a = hermitian_eigh(torch.from_numpy(np.stack([b[0] for b in blocks])).to("cuda"))
    eig_b = hermitian_eigh(torch.from_numpy(np.stack([b[1] for b in blocks])).to("cuda"))
    stream = _lib.stream_handle()
    for row in range(len(hamiltonians)):
        spec_a = _Spectrum(torch, eig_a[0][row], eig_a[1][row])
        spec_b = _Spectrum(torch, eig_b[0][row], eig_b[1][row])
        margin = 3
        half_a = int(math.ceil(spec_a.max_gap / delta)) + margin
        half_b = int(math.ceil(spec_b.max_gap / delta)) + margin
        out_len = (2 * half_a + 1) + (2 * half_b + 1) - 1
        nfft = 1 << max(1, (out_len - 1).bit_length())
        # rows 0..8: radical A's binned spectra of (p, q), rows 9..17: radical B's, zero-padded
        rows = torch.zeros((18, nfft), dtype=torch.complex128, device="cuda")
        for p in range(3):
            for q in range(3):
                ga = _binned(torch, spec_a, p, q, delta, half_a, bad)
                gb = _binned(torch, spec_b, p, q, delta, half_b, bad)
                rows[3 * p + q, :ga.numel()] = ga
                rows[9 + 3 * p + q, :gb.numel()] = gb
        if int(bad.item()):
            raise ValueError("Frequency grid is too small for transition spectrum.")
        scratch = torch.empty_like(rows)
        _lib.call("rpm_fft_pow2", nfft, 18, _lib.ptr(rows), _lib.ptr(scratch), 0, stream)
        combined = torch.zeros((1, nfft), dtype=torch.complex128, device="cuda")
        for k in range(9):
            _lib.call("rpm_spectrum_mac", nfft, _lib.ptr(combined), _lib.ptr(rows[k]), _lib.ptr(rows[9 + k]), stream)
        _lib.call("rpm_fft_pow2", nfft, 1, _lib.ptr(combined), _lib.ptr(scratch), 1, stream)
        conv = combined[0, :out_len] / nfft
        omega = (torch.arange(out_len, dtype=torch.float64, device="cuda") - (half_a + half_b)) * delta
        initial[row] = float((0.25 + conv.sum()).real.item())
        for col, tau in enumerate(lifetimes):
            k = 1.0 / tau
            kern = k / (k - 1j * omega)
            yields[row, col] = float((0.25 + (conv * kern).sum()).real.item())
    return yields, initial
