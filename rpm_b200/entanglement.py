"""Stored-state entanglement observables on the GPU (poster_reproduction/core.py:311-365).

Every observable here is a function of the reduced density matrix of one
side of a bipartition, rho_A = M M^H with M the state reshaped to
(kept part) x (traced part).  rho_A is formed on the GPU by the library's
``rpm_reduced_density`` kernels (FP64) and diagonalised by the library's
batched FP64 Hermitian eigen-solver (``rpm_he_eigh``; at most the smaller
side's dimension); the Schmidt
coefficients are then the row norms of U^H M (``rpm_schmidt_norms``), which
resolves small coefficients to ~eps |M| where square roots of rho_A's
eigenvalues would only resolve ~sqrt(eps).  States may be one vector or a batch
(rows), as NumPy arrays or CUDA tensors; every function returns NumPy
values.

* ``pure_log_negativity(state, dimensions, left_axes)``: 2 log2 of the sum of
  the normalised Schmidt coefficients (core.py:311-328); the smaller side of
  the split is kept, the Schmidt spectrum does not depend on which.
* ``reduced_electron_density(state, dimensions)``: the hermitised 4 x 4
  density matrix of the electron pair (axes 0, 1) (core.py:331-334).
* ``partial_transpose_two_qubits``, ``mixed_two_electron_log_negativity``,
  ``mixed_two_electron_log_negativity_batch`` (core.py:337-365).
* ``entanglement_cell(...)``: the reference's Fig. 9 cell
  (runner.py:263-292) on the plain FP64 GPU path.
"""

from __future__ import annotations

import math
from typing import Sequence

import numpy as np

from . import _lib
from .engine import _torch
from .factorized import hermitian_eigh


def _offsets(dimensions: Sequence[int], axes: Sequence[int]) -> np.ndarray:
    """Memory offsets of the mixed-radix index over ``axes`` (first slowest)."""
    dims = tuple(int(v) for v in dimensions)
    strides = [1] * len(dims)
    for k in range(len(dims) - 2, -1, -1):
        strides[k] = strides[k + 1] * dims[k + 1]
    off = np.zeros(1, dtype=np.int64)
    for a in axes:
        off = (off[:, None] + np.arange(dims[a], dtype=np.int64)[None, :] * strides[a]).reshape(-1)
    return off


def _as_batch(states, n: int):
    torch = _torch()
    if isinstance(states, torch.Tensor):
        x = states.to(device="cuda", dtype=torch.complex128)
    else:
        x = torch.from_numpy(np.ascontiguousarray(np.asarray(states, dtype=np.complex128))).to("cuda")
    single = x.dim() == 1
    x = x.reshape(1, -1) if single else x.reshape(x.shape[0], -1)
    if x.shape[1] != n:
        raise ValueError(f"State dimension {x.shape[1]} does not match {n}.")
    return x.contiguous(), single


def reduced_density(states, dimensions: Sequence[int], kept_axes: Sequence[int]):
    """rho_A = M M^H for the kept axes, (batch, dA, dA) complex128 CUDA tensor."""
    torch = _torch()
    dims = tuple(int(v) for v in dimensions)
    kept = tuple(int(a) for a in kept_axes)
    rest = tuple(a for a in range(len(dims)) if a not in kept)
    n = math.prod(dims)
    x, _ = _as_batch(states, n)
    offa = torch.from_numpy(_offsets(dims, kept)).to("cuda")
    offc = torch.from_numpy(_offsets(dims, rest)).to("cuda")
    da = int(offa.numel())
    rho = torch.empty((x.shape[0], da, da), dtype=torch.complex128, device="cuda")
    batch = 65535
    for s0 in range(0, x.shape[0], batch):
        xs = x[s0:s0 + batch]
        _lib.call("rpm_reduced_density", _lib.ptr(xs), int(xs.shape[0]), int(n), _lib.ptr(offa), da, _lib.ptr(offc),
                  int(offc.numel()), _lib.ptr(rho[s0:s0 + batch]), _lib.stream_handle())
    return rho


def pure_log_negativity(state, dimensions: Sequence[int], left_axes: Sequence[int]):
    """Log negativity of a pure state across ``left_axes`` | rest (core.py:311-328)."""
    torch = _torch()
    dims = tuple(int(v) for v in dimensions)
    left = tuple(int(v) for v in left_axes)
    if len(set(left)) != len(left) or any(axis < 0 or axis >= len(dims) for axis in left):
        raise ValueError("Invalid subsystem axes.")
    right = tuple(a for a in range(len(dims)) if a not in left)
    dl = math.prod(dims[a] for a in left)
    dr = math.prod(dims[a] for a in right)
    kept = left if dl <= dr else right
    rest = tuple(a for a in range(len(dims)) if a not in kept)
    x, single = _as_batch(state, math.prod(dims))
    rho = reduced_density(x, dims, kept)
    _, vec = hermitian_eigh(rho)  # the library's FP64 eigen-solver
    vec = vec.contiguous()
    # Schmidt norms |U^H M| row by row (accurate for small Schmidt values)
    offa = torch.from_numpy(_offsets(dims, kept)).to("cuda")
    offc = torch.from_numpy(_offsets(dims, rest)).to("cuda")
    da = int(offa.numel())
    sigma2 = torch.empty((x.shape[0], da), dtype=torch.float64, device="cuda")
    for s0 in range(0, x.shape[0], 65535):
        xs = x[s0:s0 + 65535]
        _lib.call("rpm_schmidt_norms", _lib.ptr(xs), int(xs.shape[0]), int(x.shape[1]), _lib.ptr(offa), da,
                  _lib.ptr(offc), int(offc.numel()), _lib.ptr(vec[s0:s0 + 65535]), _lib.ptr(sigma2[s0:s0 + 65535]),
                  _lib.stream_handle())
    norm2 = sigma2.sum(dim=-1)
    if bool((norm2 == 0.0).any()):
        raise ValueError("Cannot evaluate entanglement of the zero state.")
    values = 2.0 * torch.log2(sigma2.sqrt().sum(dim=-1) / norm2.sqrt())
    out = values.cpu().numpy()
    return float(out[0]) if single else out


def reduced_electron_density(state, dimensions: Sequence[int]):
    """Hermitised 4 x 4 reduced density matrix of the electron pair (core.py:331-334)."""
    dims = tuple(int(v) for v in dimensions)
    x, single = _as_batch(state, math.prod(dims))
    rho = reduced_density(x, dims, (0, 1))
    rho = 0.5 * (rho + rho.conj().transpose(-1, -2))
    out = rho.cpu().numpy()
    return out[0] if single else out


def partial_transpose_two_qubits(rho, subsystem: int = 0) -> np.ndarray:
    """Partial transpose of a 4 x 4 two-qubit density matrix (core.py:337-345)."""
    tensor = np.asarray(rho, dtype=complex).reshape(2, 2, 2, 2)
    if subsystem == 0:
        tensor = tensor.transpose(2, 1, 0, 3)
    elif subsystem == 1:
        tensor = tensor.transpose(0, 3, 2, 1)
    else:
        raise ValueError("subsystem must be 0 or 1.")
    return tensor.reshape(4, 4)


def mixed_two_electron_log_negativity_batch(rho) -> np.ndarray:
    """Two-qubit log negativity over any leading axes (core.py:354-365), on the GPU."""
    torch = _torch()
    matrices = np.asarray(rho, dtype=complex)
    if matrices.shape[-2:] != (4, 4):
        raise ValueError("rho must end in shape (4, 4).")
    leading = matrices.shape[:-2]
    m = torch.from_numpy(np.ascontiguousarray(matrices.reshape(-1, 4, 4))).to("cuda")
    herm = 0.5 * (m + m.conj().transpose(-1, -2))
    partial = herm.reshape(-1, 2, 2, 2, 2).permute(0, 3, 2, 1, 4).reshape(-1, 4, 4)
    lam, _ = hermitian_eigh(partial.contiguous())
    values = torch.clamp(torch.log2(lam.abs().sum(dim=-1)), min=0.0)
    return values.cpu().numpy().reshape(leading)


def mixed_two_electron_log_negativity(rho) -> float:
    """Two-qubit log negativity of one 4 x 4 density matrix (core.py:348-351)."""
    return float(mixed_two_electron_log_negativity_batch(np.asarray(rho)[None])[0])


def entanglement_cell(nuclear_count: int, theta_deg: float, field_mT: float, sample_id: int, master_seed: int,
                      *, coupling=None, quadrupole_scale: float | None = None) -> dict:
    """The reference's entanglement cell (runner.py:263-292) on the plain FP64 GPU path.

    A product-basis nuclear state paired with the electron singlet is
    propagated on the entanglement grid with every state stored on the GPU;
    the radical | radical and electron | nuclei log negativities and the
    electron density are evaluated for every stored state.
    """
    from .engine import singlet_population
    from .production import (PRODUCTION_COUPLING, build_hamiltonian, dimensions_for, entanglement_time_grids_us,
                             full_product_basis_indices, make_propagator, paired_product_indices,
                             product_basis_initial_state, selected_nuclei, selected_radicals)

    kwargs = {} if quadrupole_scale is None else {"quadrupole_scale": quadrupole_scale}
    nuclei = selected_nuclei(int(nuclear_count))
    h = build_hamiltonian(float(theta_deg), float(field_mT), coupling=coupling or PRODUCTION_COUPLING, nuclei=nuclei,
                          radicals=selected_radicals(int(nuclear_count)), **kwargs)
    dims = dimensions_for(nuclei)
    indices = paired_product_indices(int(nuclear_count), full_product_basis_indices(master_seed, sample_id))
    initial = product_basis_initial_state(dims, indices)
    times, _ = entanglement_time_grids_us()
    result = make_propagator(h).propagate(initial, times, lambda s: singlet_population(s, dims), store_states=True)
    per_radical = int(nuclear_count) // 2
    radical_left = (0,) + tuple(range(2, 2 + per_radical))
    radical = pure_log_negativity(result.states, dims, radical_left)
    electron_nuclear = pure_log_negativity(result.states, dims, (0, 1))
    rho = reduced_electron_density(result.states, dims)
    return {
        "times_us": times,
        "radical_log_negativity": np.asarray(radical),
        "electron_nuclear_log_negativity": np.asarray(electron_nuclear),
        "electron_density_real": rho.real,
        "electron_density_imag": rho.imag,
        "initial_radical_log_negativity": np.array(np.asarray(radical)[0]),
        "initial_electron_nuclear_log_negativity": np.array(np.asarray(electron_nuclear)[0]),
        "singlet_population": result.observable_values,
    }
