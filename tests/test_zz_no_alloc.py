"""The allocation-free H psi entry point, called through the C ABI.

rpm_hpsi_noalloc is for callers that may not call cudaMalloc while they run
(for example a framework whose run loop owns all device memory through its own
pool, where a cudaMalloc would synchronise the device and escape the pool's
accounting).  It keeps its scratch in a fixed 4 MiB array compiled into the
library and picks the same kernels as rpm_hpsi.  This file is named so that
pytest collects it last.
"""

import ctypes
import math

import pytest

pytestmark = pytest.mark.gpu

REL_TOL = {128: 1e-13, 64: 2e-6}  # the tolerances of the other H psi tests


def _entry():
    from rpm_b200 import _lib

    lib = _lib.load()
    fn = lib.rpm_hpsi_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong,
                   ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return lib, fn


@pytest.mark.parametrize("precision,batch", [(128, 1), (64, 2)])
def test_noalloc_matches_allocating_entry_point(precision, batch):
    import torch

    import rpm_b200 as rb
    from rpm_b200 import _lib, synthetic

    lib, fn = _entry()
    full = synthetic.full_system()
    h = rb.CompiledFullPairHamiltonian(full.dimensions, full.terms(math.pi / 4, 0.3), left_axes=full.left_axes,
                                       right_axes=full.right_axes)
    n = h.dimension
    dtype = torch.complex128 if precision == 128 else torch.complex64
    x = torch.from_numpy(synthetic.random_phase_vectors(full.dimensions, batch, 31)).to("cuda", dtype)
    expected = torch.empty_like(x)
    h.apply(x, expected, batch=batch, precision=precision)  # rpm_hpsi, cudaMalloc'd scratch
    stream = _lib.stream_handle()
    for _ in range(2):  # two calls in a row reuse the same static scratch
        out = torch.full_like(x, float("nan"))
        status = fn(h._system.handle, precision, _lib.ptr(x), _lib.ptr(out), batch, n, stream)
        assert status == 0, lib.rpm_last_error().decode()
        torch.cuda.synchronize()
        rel = float(torch.linalg.vector_norm(out - expected) / torch.linalg.vector_norm(expected))
        assert rel < REL_TOL[precision]


def test_noalloc_rejects_batches_beyond_its_scratch():
    import torch

    import rpm_b200 as rb
    from rpm_b200 import _lib, synthetic

    lib, fn = _entry()
    full = synthetic.full_system()
    h = rb.CompiledFullPairHamiltonian(full.dimensions, full.terms(0.2, 0.0), left_axes=full.left_axes,
                                       right_axes=full.right_axes)
    n = h.dimension
    x = torch.zeros((2, n), dtype=torch.complex128, device="cuda")  # 2 x 3.5 MB > 4 MiB
    out = torch.empty_like(x)
    status = fn(h._system.handle, 128, _lib.ptr(x), _lib.ptr(out), 2, n, _lib.stream_handle())
    assert status == _lib.RPM_E_UNSUPPORTED
    assert "4 MiB" in lib.rpm_last_error().decode()


def _small_variant(kind):
    """A 96-dimensional system that takes one kernel route of rpm_hpsi:
    'csr' (a radical term coupling two nuclei: CSR passes), 'unequal'
    (unequal recombination rates: the non-Hermitian pair operator on the cube
    passes) or 'generic' (a cross-radical nuclear term: no radical split, the
    per-term kernel)."""
    import numpy as np

    import rpm_b200 as rb
    from rpm_b200 import synthetic

    small = synthetic.small_system()
    terms = list(small.terms(0.4, 0.9))
    rng = np.random.default_rng(8)
    left, right = small.left_axes[1:], small.right_axes[1:]
    if kind == "unequal":
        h = rb.CompiledFullPairHamiltonian(small.dimensions, terms, left_axes=small.left_axes,
                                           right_axes=small.right_axes)
        h.set_recombination_rates(1.0, 2.0)
        return h, small.dimensions
    if kind == "csr":
        axes = tuple(left[:2]) if len(left) >= 2 else tuple(right[:2])
    else:
        axes = (left[0], right[0])
    d = small.dimensions[axes[0]] * small.dimensions[axes[1]]
    a = rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d))
    terms.append(rb.LocalTerm(axes, 0.3 * (a + a.conj().T)))
    return rb.MatrixFreeHamiltonian(small.dimensions, terms), small.dimensions


@pytest.mark.parametrize("kind", ["csr", "unequal", "generic"])
@pytest.mark.parametrize("precision", [128, 64])
def test_noalloc_takes_every_route_of_the_allocating_entry_point(kind, precision):
    import torch

    from rpm_b200 import _lib, synthetic

    lib, fn = _entry()
    h, dims = _small_variant(kind)
    n = h.dimension
    batch = 3
    dtype = torch.complex128 if precision == 128 else torch.complex64
    x = torch.from_numpy(synthetic.random_phase_vectors(dims, batch, 77)).to("cuda", dtype)
    expected = torch.empty_like(x)
    h.apply(x, expected, batch=batch, precision=precision)
    for _ in range(2):
        out = torch.full_like(x, float("nan"))
        status = fn(h._system.handle, precision, _lib.ptr(x), _lib.ptr(out), batch, n, _lib.stream_handle())
        assert status == 0, lib.rpm_last_error().decode()
        torch.cuda.synchronize()
        rel = float(torch.linalg.vector_norm(out - expected) / torch.linalg.vector_norm(expected))
        assert rel < REL_TOL[precision]
