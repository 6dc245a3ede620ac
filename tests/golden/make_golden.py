"""Generate golden fixtures by running the reference implementation itself.

Run once in a checkout that has the reference next to it:

    python tests/golden/make_golden.py <RPM checkout>

It imports ``rpm_statevector_engine`` / ``rpm_quantum_needle_model`` /
``poster_reproduction.core`` / ``rpm_quantum_needle_jd_sweeps`` from the
reference's ``Realistic system size/code`` directory (a stand-in
``matplotlib`` module is placed in ``sys.modules`` because those modules import
it at module level; nothing is plotted) and writes small ``.npz``/``.json``
fixtures next to this script.  Tests only read the fixtures; the reference
is not needed at test time.
"""

from __future__ import annotations

import csv
import json
import math
import sys
import time
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))


def _stub_matplotlib():
    mpl = types.ModuleType("matplotlib")
    mpl.use = lambda *a, **k: None
    pyplot = types.ModuleType("matplotlib.pyplot")
    pyplot.__getattr__ = lambda name: (lambda *a, **k: None)
    mpl.pyplot = pyplot
    backends = types.ModuleType("matplotlib.backends")
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", pyplot)
    sys.modules.setdefault("matplotlib.backends", backends)


def load_reference(root: Path):
    code = root / "Realistic system size" / "code"
    sys.path.insert(0, str(code))
    _stub_matplotlib()
    import rpm_quantum_needle_model as MOD  # noqa: N812
    import rpm_statevector_engine as ENG  # noqa: N812
    import rpm_quantum_needle_jd_sweeps as JD  # noqa: N812
    from poster_reproduction import core as CORE  # noqa: N812

    return ENG, MOD, JD, CORE


def terms_to_arrays(terms):
    axes = np.full((len(terms), 4), -1, dtype=np.int32)
    sizes = np.zeros(len(terms), dtype=np.int32)
    ops = []
    for k, t in enumerate(terms):
        axes[k, : len(t.axes)] = t.axes
        op = np.asarray(t.operator, dtype=complex)
        sizes[k] = op.shape[0]
        ops.append(op.reshape(-1))
    return axes, sizes, np.concatenate(ops)


def ref_terms(ENG, ours):
    return [ENG.LocalTerm(tuple(t.axes), np.asarray(t.operator, dtype=complex), t.label) for t in ours]


def sample_indices(n, count, seed):
    return np.sort(np.random.default_rng(seed).choice(n, size=min(count, n), replace=False))


def checksums(vec, seed, count=256):
    rng = np.random.default_rng(seed)
    probe = rng.normal(size=vec.size) + 1j * rng.normal(size=vec.size)
    idx = sample_indices(vec.size, count, seed + 1)
    return {
        "norm2": float(np.vdot(vec, vec).real),
        "probe_dot": np.vdot(probe, vec),
        "sample_idx": idx,
        "sample_val": vec[idx],
    }


def main(root: Path) -> None:
    ENG, MOD, JD, CORE = load_reference(root)
    from rpm_b200 import synthetic

    out: dict[str, np.ndarray] = {}
    t0 = time.time()

    # --- spin algebra and local operators ----------------------------------
    for s in (0.5, 1.0, 1.5):
        ops = MOD.spin_operators(s)
        for name, op in zip("xyz", ops):
            out[f"spin_{s}_{name}"] = op
    rng = np.random.default_rng(7)
    t3 = rng.normal(size=(3, 3))
    out["coupling_tensor"] = t3
    out["coupling_half_one"] = ENG.two_spin_coupling_operator(0.5, 1.0, t3)
    out["coupling_half_half"] = ENG.two_spin_coupling_operator(0.5, 0.5, t3)
    q = 0.5 * (t3 + t3.T)
    out["quad_tensor"] = q
    out["quad_one"] = ENG.quadrupole_operator(1.0, q)
    out["eh_axis"] = np.array([0.3, -0.4, 0.8])
    out["eh_op"] = ENG.efimova_hore_electron_coupling_operator(1.7, -2.3, out["eh_axis"])
    for key, tensor in MOD.QUADRUPOLE_TENSORS_MT.items():
        out[f"qtensor_{key}"] = tensor
    for k, nuc in enumerate(MOD.ALL_NUCLEI):
        out[f"hf_{k}"] = nuc.tensor_mT
    out["field_vec"] = MOD.field_vector_mT(37.0, 50.0)

    # --- seeds and initial states -------------------------------------------
    out["seeds"] = np.array([JD._seed(20260731, s) for s in range(4)], dtype=np.uint64)
    init = CORE.random_phase_initial_state(MOD.SYSTEM_DIMENSIONS, 20260731, 0)
    out["init_s0_checks_idx"] = sample_indices(init.size, 64, 3)
    out["init_s0_checks_val"] = init[out["init_s0_checks_idx"]]

    # --- Simpson quadrature ---------------------------------------------------
    import scipy.integrate

    for n in (1, 2, 3, 4, 5, 8, 9, 4001):
        x = np.sort(rng.uniform(0, 3, n)) if n < 100 else np.arange(n) * 0.00125
        y = rng.normal(size=n)
        out[f"simpson_x_{n}"] = x
        out[f"simpson_y_{n}"] = y
        out[f"simpson_v_{n}"] = np.array(float(scipy.integrate.simpson(y, x=x)) if n > 1 else 0.0)
    tt = np.arange(4001) * 0.00125
    pp = 0.25 + 0.1 * np.cos(3 * tt)
    out["yield_t"] = tt
    out["yield_p"] = pp
    out["yield_v"] = np.array(JD.integrate_yield(tt, pp, 1.0))

    # --- small synthetic system (dim 96) --------------------------------------
    small = synthetic.small_system()
    terms = small.terms(0.0, 0.0)
    ax, sz, ops = terms_to_arrays(terms)
    out["small_dims"] = np.array(small.dimensions)
    out["small_left"] = np.array(small.left_axes)
    out["small_right"] = np.array(small.right_axes)
    out["small_axes"], out["small_sizes"], out["small_ops"] = ax, sz, ops
    h_generic = ENG.MatrixFreeHamiltonian(small.dimensions, ref_terms(ENG, terms))
    h_split = ENG.CompiledFullPairHamiltonian(small.dimensions, ref_terms(ENG, terms), left_axes=small.left_axes,
                                              right_axes=small.right_axes)
    out["small_dense"] = h_generic.explicit_matrix()
    vec = rng.normal(size=96) + 1j * rng.normal(size=96)
    out["small_vec"] = vec
    out["small_hvec"] = h_generic.matvec(vec)
    out["small_hvec_split"] = h_split.matvec(vec)
    psi0 = synthetic.random_phase_vectors(small.dimensions, 2, 11)
    out["small_psi0"] = psi0
    times = np.arange(0, 401) * 0.00125  # 0 .. 0.5 us
    out["small_times"] = times
    for tag, knobs in {
        "default": {},
        "cfg0": dict(minimum_dimension=30, maximum_dimension=30, state_error_budget=1e-10),
        "cfg1": dict(minimum_dimension=8, maximum_dimension=40, state_error_budget=1e-10),
    }.items():
        prop = ENG.AdaptiveLanczosPropagator(h_split, **knobs)
        res = prop.propagate(psi0[0], times, ENG.SingletPopulationObservable(small.dimensions))
        out[f"small_{tag}_values"] = res.observable_values
        out[f"small_{tag}_bounds"] = res.observable_error_bounds
        out[f"small_{tag}_state_errors"] = res.state_error_estimates
        out[f"small_{tag}_final"] = res.final_state
        s = res.stats
        out[f"small_{tag}_stats"] = np.array([s.accepted_steps, s.rejected_steps, s.matvecs,
                                              s.maximum_krylov_dimension, s.minimum_step_us, s.maximum_step_us,
                                              s.accumulated_state_error, s.maximum_norm_error])
        out[f"small_{tag}_yield"] = np.array(JD.integrate_yield(times, res.observable_values, 1.0))
    # direct (callable) observable path with stored states
    prop = ENG.AdaptiveLanczosPropagator(h_split, minimum_dimension=8, maximum_dimension=16,
                                         state_error_budget=1e-9)
    res = prop.propagate(psi0[1], times[:41], lambda v: float(abs(v[5]) ** 2), store_states=True)
    out["small_direct_values"] = res.observable_values
    out["small_direct_states"] = res.states
    out["small_direct_stats"] = np.array([res.stats.accepted_steps, res.stats.rejected_steps, res.stats.matvecs])

    # --- prefix systems (6 and 10 nuclei) ------------------------------------
    full = synthetic.full_system()
    for per in (3, 5):
        sub = synthetic.prefix_system(full, per)
        t_sub = sub.terms(0.7, 1.1)
        ax, sz, ops = terms_to_arrays(t_sub)
        key = f"prefix{2 * per}"
        out[f"{key}_dims"] = np.array(sub.dimensions)
        out[f"{key}_left"] = np.array(sub.left_axes)
        out[f"{key}_right"] = np.array(sub.right_axes)
        out[f"{key}_axes"], out[f"{key}_sizes"], out[f"{key}_ops"] = ax, sz, ops
        h = ENG.CompiledFullPairHamiltonian(sub.dimensions, ref_terms(ENG, t_sub), left_axes=sub.left_axes,
                                            right_axes=sub.right_axes)
        v = synthetic.random_phase_vectors(sub.dimensions, 1, 5)[0]
        out[f"{key}_psi0"] = v
        hv = h.matvec(v)
        out[f"{key}_hvec"] = hv if hv.size <= 1000 else np.array([])
        for name, val in checksums(hv, 99).items():
            out[f"{key}_hvec_{name}"] = val
        tgrid = np.arange(0, 81) * 0.00125
        prop = ENG.AdaptiveLanczosPropagator(h, minimum_dimension=8, maximum_dimension=40, state_error_budget=1e-10)
        res = prop.propagate(v, tgrid, ENG.SingletPopulationObservable(sub.dimensions))
        out[f"{key}_times"] = tgrid
        out[f"{key}_values"] = res.observable_values
        out[f"{key}_state_errors"] = res.state_error_estimates
        out[f"{key}_stats"] = np.array([res.stats.accepted_steps, res.stats.rejected_steps, res.stats.matvecs,
                                        res.stats.maximum_krylov_dimension])
        for name, val in checksums(res.final_state, 123).items():
            out[f"{key}_final_{name}"] = val
        print(f"{key}: dim {sub.dimension} done at {time.time() - t0:.1f}s", flush=True)

    # --- full size: synthetic system and production Hamiltonian ---------------
    t_full = full.terms(math.pi / 4, 0.0)
    ax, sz, ops = terms_to_arrays(t_full)
    out["full_axes"], out["full_sizes"], out["full_ops"] = ax, sz, ops
    h = ENG.CompiledFullPairHamiltonian(full.dimensions, ref_terms(ENG, t_full), left_axes=full.left_axes,
                                        right_axes=full.right_axes)
    v = synthetic.random_phase_vectors(full.dimensions, 1, 2024)[0]
    hv = h.matvec(v)
    for name, val in checksums(hv, 7).items():
        out[f"full_hvec_{name}"] = val
    h_prod = CORE.build_hamiltonian(0.0, 0.05, model=CORE.PRODUCTION_MODEL)
    hv = h_prod.matvec(init)
    for name, val in checksums(hv, 8).items():
        out[f"prod_hvec_{name}"] = val
    tgrid = np.arange(0, 9) * 0.00125  # 0 .. 0.01 us
    prop = CORE.make_propagator(h_prod)
    res = prop.propagate(init, tgrid, ENG.SingletPopulationObservable(MOD.SYSTEM_DIMENSIONS))
    out["prod_times"] = tgrid
    out["prod_values"] = res.observable_values
    out["prod_state_errors"] = res.state_error_estimates
    out["prod_stats"] = np.array([res.stats.accepted_steps, res.stats.rejected_steps, res.stats.matvecs,
                                  res.stats.maximum_krylov_dimension])
    for name, val in checksums(res.final_state, 321).items():
        out[f"prod_final_{name}"] = val
    print(f"full size done at {time.time() - t0:.1f}s", flush=True)

    np.savez_compressed(HERE / "reference_golden.npz", **out)

    # --- archived full-size production yields (results CSV) ------------------
    rows = list(csv.DictReader(open(root / "results" / "quadrupole" / "full14_uncoupled_tau5_29angles"
                                    / "raw_sample_yields.csv")))
    keep = []
    for r in rows:
        if int(r["sample_id"]) == 0 and float(r["theta_deg"]) in (0.0, 90.0):
            keep.append({k: r[k] for k in ("electron_interactions", "scale", "theta_deg", "sample_id", "yield",
                                           "quadrature_error", "yield_propagation_estimate", "yield_tail_bound")})
    (HERE / "archived_full14_yields.json").write_text(json.dumps(keep, indent=1) + "\n")
    print(f"wrote fixtures in {time.time() - t0:.1f}s")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(f"usage: python {Path(__file__).name} <path of the RPM checkout>")
    main(Path(sys.argv[1]))
