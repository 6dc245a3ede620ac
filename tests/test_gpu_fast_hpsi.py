"""Shape-specialised complex64 H psi against complex128 and the general cube kernels (GPU).

Bars: complex64 action within 2e-6 relative of the complex128 action (FP32
storage and accumulation); within 1e-6 relative of the general complex64
cube kernels; the fused <psi, H psi> of a batched launch within 1e-6 relative.
"""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL64 = 2e-6
REL_CUBE = 1e-6


@pytest.fixture(scope="module")
def rb():
    import rpm_b200

    return rpm_b200


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


def _systems(rb):
    from rpm_b200 import synthetic

    full = synthetic.full_system()
    out = []
    for name, sys_, th, ph in (("full", full, math.pi / 4, 0.0), ("full_oblique", full, 1.1, 2.3),
                               ("prefix10", synthetic.prefix_system(full, 5), 0.4, 0.9)):
        h = rb.CompiledFullPairHamiltonian(sys_.dimensions, sys_.terms(th, ph), left_axes=sys_.left_axes,
                                           right_axes=sys_.right_axes)
        out.append((name, sys_, h))
    out.append(("production", None, rb.build_hamiltonian(0.7, 0.05)))
    return out


def _apply64(rb, h, vecs, ld):
    import torch

    n = h.dimension
    x = torch.zeros((len(vecs), ld), dtype=torch.complex64, device="cuda")
    for k, v in enumerate(vecs):
        x[k, :n] = torch.from_numpy(v.astype(np.complex64))
    y = torch.zeros_like(x)
    from rpm_b200 import _lib

    _lib.call("rpm_hpsi", h._system.handle, _lib.PREC_C64, _lib.ptr(x), _lib.ptr(y), len(vecs), ld,
              _lib.stream_handle())
    torch.cuda.synchronize()
    return y[:, :n].cpu().numpy()


@pytest.mark.parametrize("idx", [0, 1, 2, 3])
def test_fast_action_matches_fp64_and_cube(rb, idx):
    from rpm_b200 import _lib

    name, _, h = _systems(rb)[idx]
    assert h._system.fast_hpsi, f"{name}: shape-specialised kernels not selected"
    rng = np.random.default_rng(11 + idx)
    n = h.dimension
    vecs = [rng.normal(size=n) + 1j * rng.normal(size=n) for _ in range(3)]
    ld = n + 64
    fast = _apply64(rb, h, vecs, ld)
    _lib.call("rpm_set_cube_tuning", 2, 2, 4, 8)
    try:
        cube = _apply64(rb, h, vecs, ld)
    finally:
        _lib.call("rpm_set_cube_tuning", 0, 0, 0, 0)
    for k, v in enumerate(vecs):
        ref = h.matvec(v)
        assert _rel(fast[k], ref) < REL64, name
        assert _rel(fast[k], cube[k]) < REL_CUBE, name


def test_fast_path_not_claimed_for_other_axis_orders(rb):
    from rpm_b200 import synthetic

    small = synthetic.small_system()  # too few spin-1/2 digits per radical
    h = rb.CompiledFullPairHamiltonian(small.dimensions, small.terms(0.3, 0.0), left_axes=small.left_axes,
                                       right_axes=small.right_axes)
    assert not h._system.fast_hpsi
    full = synthetic.full_system()
    # the same Hamiltonian with the two electron axes swapped: no standard layout
    terms = full.terms(0.5, 0.0)
    perm = {0: 1, 1: 0}
    swapped = [rb.LocalTerm(tuple(perm.get(a, a) for a in t.axes), t.operator, t.label) for t in terms]
    assert any(t.axes == (1, 0) for t in swapped)
    h2 = rb.CompiledFullPairHamiltonian(full.dimensions, swapped, left_axes=(1,) + full.left_axes[1:],
                                        right_axes=(0,) + full.right_axes[1:], electron_pair_axes=(1, 0))
    assert not h2._system.fast_hpsi
    v = synthetic.random_phase_vectors(full.dimensions, 1, 5)[0]
    assert _rel(_apply64(rb, h2, [v], full.dimension)[0], h2.matvec(v)) < REL64


@pytest.mark.parametrize("idx", [0, 2, 3])
def test_complex128_fast_passes_match_general_cube_kernels(rb, idx):
    """complex128 H psi on the shape-specialised passes (the default for the standard layout) against the
    general cube kernels (forced through the tuning hook), batched, with a strided leading dimension."""
    import torch

    from rpm_b200 import _lib

    name, _, h = _systems(rb)[idx]
    n = h.dimension
    ld = n + 64
    rng = np.random.default_rng(17 + idx)
    x = torch.zeros((3, ld), dtype=torch.complex128, device="cuda")
    x[:, :n] = torch.from_numpy(rng.normal(size=(3, n)) + 1j * rng.normal(size=(3, n)))
    fast, general = torch.zeros_like(x), torch.zeros_like(x)
    _lib.call("rpm_hpsi", h._system.handle, _lib.PREC_C128, _lib.ptr(x), _lib.ptr(fast), 3, ld, _lib.stream_handle())
    try:
        _lib.call("rpm_set_cube_tuning", 2, 2, 0, 0)  # any explicit choice bypasses the specialised passes
        _lib.call("rpm_hpsi", h._system.handle, _lib.PREC_C128, _lib.ptr(x), _lib.ptr(general), 3, ld,
                  _lib.stream_handle())
    finally:
        _lib.call("rpm_set_cube_tuning", 0, 0, 0, 0)
    torch.cuda.synchronize()
    assert h._system.fast_hpsi
    for b in range(3):
        assert _rel(fast[b, :n].cpu().numpy(), general[b, :n].cpu().numpy()) < 1e-13, name
