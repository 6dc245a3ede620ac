"""Golden fixtures of the reference's entanglement observables (core.py:107-365).

Run once with the reference next to the checkout:

    python tests/golden/make_entanglement_golden.py <RPM checkout>

It runs the reference's own ``poster_reproduction.core`` functions (through
``make_golden.load_reference``) on seeded random states of a 4-nucleus paired
prefix and on a short entanglement-cell propagation of the same prefix,
and writes ``entanglement_golden.npz`` next to this script.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

from make_golden import load_reference  # noqa: E402


def main(root: Path) -> None:
    ENG, MOD, JD, CORE = load_reference(root)  # noqa: N806
    out = {}
    fine, idx = CORE.entanglement_time_grids_us()
    out["grid_fine"], out["grid_coarse_idx"] = fine, idx
    out["product_indices"] = np.array([CORE.full_product_basis_indices(CORE.MASTER_SEED, s) for s in range(4)])
    # random states on the 4-nucleus paired prefix
    nuclei = CORE.selected_nuclei(4)
    dims = CORE.dimensions_for(nuclei)
    out["dims4"] = np.array(dims)
    rng = np.random.default_rng(4242)
    n = int(np.prod(dims))
    states = rng.normal(size=(5, n)) + 1j * rng.normal(size=(5, n))
    states[0] = CORE.product_basis_initial_state(
        dims, CORE.paired_product_indices(4, CORE.full_product_basis_indices(CORE.MASTER_SEED, 3)))
    out["states4"] = states
    splits = {"radical": (0,) + tuple(range(2, 2 + 2)), "electrons": (0, 1), "axis3": (3,), "mixed": (1, 2, 5)}
    for name, left in splits.items():
        out[f"lneg_{name}"] = np.array([CORE.pure_log_negativity(s, dims, left) for s in states])
    rho = np.array([CORE.reduced_electron_density(s, dims) for s in states])
    out["rho_electrons"] = rho
    out["mixed_lneg"] = CORE.mixed_two_electron_log_negativity_batch(rho / np.trace(rho, axis1=1, axis2=2)[:, None, None])
    out["pt0"] = CORE.partial_transpose_two_qubits(rho[1], 0)
    out["pt1"] = CORE.partial_transpose_two_qubits(rho[1], 1)
    # a short entanglement-cell propagation (4 nuclei, first 0.2 us of the grid)
    nuclei2 = CORE.selected_nuclei(4)
    dims2 = CORE.dimensions_for(nuclei2)
    h = CORE.build_hamiltonian(90.0, 0.05, nuclei=nuclei2, radicals=CORE.selected_radicals(4))
    init = CORE.product_basis_initial_state(
        dims2, CORE.paired_product_indices(4, CORE.full_product_basis_indices(CORE.MASTER_SEED, 1)))
    times = fine[fine <= 0.2 + 1e-12]
    res = CORE.make_propagator(h).propagate(init, times, lambda s: ENG.singlet_population(s, dims2), store_states=True)
    out["cell_dims"] = np.array(dims2)
    out["cell_times"] = times
    out["cell_radical_lneg"] = np.array([CORE.pure_log_negativity(s, dims2, (0, 2, 3)) for s in res.states])
    out["cell_electron_lneg"] = np.array([CORE.pure_log_negativity(s, dims2, (0, 1)) for s in res.states])
    out["cell_rho"] = np.array([CORE.reduced_electron_density(s, dims2) for s in res.states])
    out["cell_singlet"] = res.observable_values
    np.savez_compressed(HERE / "entanglement_golden.npz", **out)
    print("wrote", HERE / "entanglement_golden.npz", sorted(out))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(f"usage: python {Path(__file__).name} <path of the RPM checkout>")
    main(Path(sys.argv[1]))
