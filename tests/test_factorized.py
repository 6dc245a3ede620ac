"""Factorized exact ensemble yields on the GPU against the reference (rpm_quantum_needle_reproduction.py).

Fixtures (tests/golden/factorized_golden.json) come from running the
reference's own functions (tests/golden/make_factorized_golden.py).  Bars:
the GPU FFT route within 1e-9 of the reference's FFT route (same binning;
eigenvalues and additions differ by rounding), the toy pair within the
reference self-test's 2e-4 of the exact line sum, and the initial singlet
population 1 within 1e-10.  The library's own FP64 eigen-solver, complex
products and FFTs are checked against NumPy on random inputs.
"""

import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = json.loads((Path(__file__).parent / "golden" / "factorized_golden.json").read_text())


def test_fixture_self_consistency():
    toy = GOLDEN["toy"]
    assert max(abs(a - b) for a, b in zip(toy["exact"], toy["fft"])) < 2e-4
    assert abs(toy["initial_singlet"] - 1.0) < 2e-12


@pytest.mark.gpu
@pytest.mark.parametrize("n", [2, 7, 64, 384, 576])
def test_own_hermitian_eigh_against_numpy(n):
    """Eigenvalues within 1e-12 of numpy's (relative to the spectral norm),
    residual and orthonormality of the eigenvectors at FP64 rounding, for a
    batch of two random Hermitian matrices (the radical blocks are 576 and
    384 dimensional)."""
    import torch

    from rpm_b200.factorized import hermitian_eigh

    rng = np.random.default_rng(n)
    a = rng.standard_normal((2, n, n)) + 1j * rng.standard_normal((2, n, n))
    a = 0.5 * (a + a.conj().transpose(0, 2, 1))
    lam, vec = hermitian_eigh(torch.from_numpy(a).to("cuda"))
    lam, vec = lam.cpu().numpy(), vec.cpu().numpy()
    for b in range(2):
        ref = np.linalg.eigvalsh(a[b])
        scale = np.max(np.abs(ref))
        assert np.max(np.abs(lam[b] - ref)) < 1e-12 * scale * max(1.0, n / 64)
        resid = a[b] @ vec[b] - vec[b] * lam[b][None, :]
        assert np.max(np.abs(resid)) < 1e-11 * scale * max(1.0, n / 64)
        assert np.max(np.abs(vec[b].conj().T @ vec[b] - np.eye(n))) < 1e-12 * max(1.0, n / 64)


@pytest.mark.gpu
def test_own_fft_and_products_against_numpy():
    import ctypes

    import torch

    from rpm_b200 import _lib

    rng = np.random.default_rng(5)
    n, batch = 1 << 12, 3
    x = rng.standard_normal((batch, n)) + 1j * rng.standard_normal((batch, n))
    dx = torch.from_numpy(x).to("cuda")
    scratch = torch.empty_like(dx)
    _lib.call("rpm_fft_pow2", n, batch, _lib.ptr(dx), _lib.ptr(scratch), 0, _lib.stream_handle())
    ref = np.fft.fft(x, axis=1)
    assert np.max(np.abs(dx.cpu().numpy() - ref)) < 1e-12 * np.max(np.abs(ref))
    _lib.call("rpm_fft_pow2", n, batch, _lib.ptr(dx), _lib.ptr(scratch), 1, _lib.stream_handle())
    assert np.max(np.abs(dx.cpu().numpy() / n - x)) < 1e-13 * np.max(np.abs(x))
    acc = torch.zeros_like(dx[0:1])
    _lib.call("rpm_spectrum_mac", ctypes.c_longlong(n), _lib.ptr(acc), _lib.ptr(dx[0]), _lib.ptr(dx[1]),
              _lib.stream_handle())
    assert np.max(np.abs(acc.cpu().numpy()[0] - x[0] * x[1] * n * n)) < 1e-9 * n * n
    m = 100
    a = rng.standard_normal((2, m, m)) + 1j * rng.standard_normal((2, m, m))
    b = rng.standard_normal((2, m, m)) + 1j * rng.standard_normal((2, m, m))
    da, db = torch.from_numpy(a).to("cuda"), torch.from_numpy(b).to("cuda")
    dc = torch.empty_like(da)
    _lib.call("rpm_zgemm_hn", m, 2, _lib.ptr(da), _lib.ptr(db), _lib.ptr(dc), _lib.stream_handle())
    ref = np.conj(np.transpose(a, (0, 2, 1))) @ b
    assert np.max(np.abs(dc.cpu().numpy() - ref)) < 1e-12 * np.max(np.abs(ref)) * m


@pytest.mark.gpu
def test_toy_pair_matches_reference():
    from rpm_b200.factorized import factorized_singlet_yields
    from rpm_b200.model import Nucleus
    from rpm_b200.production import UNCOUPLED, build_hamiltonian

    toy = GOLDEN["toy"]
    nuclei = (Nucleus("N", 1.0, np.diag([-0.0989, -0.0989, 1.7569])), Nucleus("N", 1.0, np.diag([0.0, 0.0, 1.0812])))
    h = build_hamiltonian(toy["theta_deg"], toy["field_uT"] / 1000.0, coupling=UNCOUPLED, nuclei=nuclei,
                          radicals=("FAD", "TrpH"))
    y, init = factorized_singlet_yields([h], toy["lifetimes"], bins_per_linewidth=toy["bins_per_linewidth"])
    np.testing.assert_allclose(y[0], toy["fft"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(y[0], toy["exact"], rtol=0, atol=2e-4)
    assert abs(init[0] - 1.0) < 1e-10


@pytest.mark.gpu
def test_full_model_matches_reference():
    from rpm_b200.factorized import factorized_singlet_yields
    from rpm_b200.production import UNCOUPLED, build_hamiltonian

    rows = GOLDEN["full"]
    hams = [build_hamiltonian(r["theta_deg"], r["field_uT"] / 1000.0, coupling=UNCOUPLED,
                              quadrupole_scale=r["quadrupole_scale"]) for r in rows]
    y, init = factorized_singlet_yields(hams, rows[0]["lifetimes"], bins_per_linewidth=rows[0]["bins_per_linewidth"])
    for k, r in enumerate(rows):
        np.testing.assert_allclose(y[k], r["yields"], rtol=0, atol=1e-9)
        assert abs(init[k] - r["initial_singlet"]) < 1e-10


@pytest.mark.gpu
def test_coupled_pair_is_rejected():
    from rpm_b200.factorized import factorized_singlet_yields
    from rpm_b200.production import build_hamiltonian

    with pytest.raises(ValueError):
        factorized_singlet_yields([build_hamiltonian(0.0, 0.05)], (1.0,))
