"""Golden fixtures of the reference's factorized ensemble yields (rpm_quantum_needle_reproduction.py).

Run once with the reference next to the checkout:

    python tests/golden/make_factorized_golden.py <RPM checkout>

Runs the reference's own ``rpm_quantum_needle_reproduction`` functions: the
toy-pair self-test (exact line sum and FFT convolution, run_self_test) and
``solve_orientation`` for three field angles of the full FAD-TrpH model at
50 uT, and writes ``factorized_golden.json`` next to this script.
"""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

from make_golden import load_reference  # noqa: E402


def main(root: Path) -> None:
    load_reference(root)
    import rpm_quantum_needle_reproduction as QN  # noqa: N812

    toy_a = QN.build_radical("X", (QN.Nucleus("N", 1.0, np.diag([-0.0989, -0.0989, 1.7569])),))
    toy_b = QN.build_radical("Y", (QN.Nucleus("N", 1.0, np.diag([0.0, 0.0, 1.0812])),))
    lifetimes = (1.0, 10.0, 100.0)
    spec_a = QN.diagonalize_radical(toy_a, 89.0, 50.0)
    spec_b = QN.diagonalize_radical(toy_b, 89.0, 50.0)
    exact = QN.direct_line_yields(spec_a, spec_b, lifetimes)
    delta = (1.0 / max(lifetimes)) / 16.0
    omega, coeff, initial = QN.convolved_correlation_spectrum(spec_a, spec_b, delta)
    fftv = QN.yields_from_spectrum(omega, coeff, lifetimes)
    out = {"toy": {"theta_deg": 89.0, "field_uT": 50.0, "lifetimes": lifetimes, "bins_per_linewidth": 16.0,
                   "exact": [exact[t] for t in lifetimes], "fft": [fftv[t] for t in lifetimes],
                   "initial_singlet": initial},
           "full": []}
    for theta in (0.0, 45.0, 90.0):
        row = QN.solve_orientation(theta, 50.0, (1.0, 5.0, 100.0), 8.0, 1.0)
        out["full"].append({"theta_deg": theta, "field_uT": 50.0, "lifetimes": [1.0, 5.0, 100.0],
                            "bins_per_linewidth": 8.0, "quadrupole_scale": 1.0,
                            "initial_singlet": row["initial_singlet"],
                            "yields": [row[f"phi_s_tau_{t:g}_us"] for t in (1.0, 5.0, 100.0)]})
    (HERE / "factorized_golden.json").write_text(json.dumps(out, indent=1))
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(f"usage: python {Path(__file__).name} <path of the RPM checkout>")
    main(Path(sys.argv[1]))
