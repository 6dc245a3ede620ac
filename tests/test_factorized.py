"""Factorized exact ensemble yields on the GPU against the reference (rpm_quantum_needle_reproduction.py).

Fixtures (tests/golden/factorized_golden.json) come from running the
reference's own functions (tests/golden/make_factorized_golden.py).  Bars:
the GPU FFT route within 1e-9 of the reference's FFT route (same binning;
eigenvalues and additions differ by rounding), the toy pair within the
reference self-test's 2e-4 of the exact line sum, and the initial singlet
population 1 within 1e-10.
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


def test_fft_length_is_smooth_and_long_enough():
    from rpm_b200.factorized import _next_fast_len

    for n in (1, 2, 11, 97, 12345, 800001):
        m = _next_fast_len(n)
        assert m >= n
        for p in (2, 3, 5, 7):
            while m % p == 0:
                m //= p
        assert m == 1


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
