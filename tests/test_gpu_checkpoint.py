"""Checkpoint cells from GPU trajectories, read back under the full-size
runner's resume checks (rpm_full14_quadrupole_experiment.py:154-194, 255-266).

A trajectory of the runner's smoke bath (FAD N5, N10, TrpH N1; D/J = -3,
Q = 1, 50 uT, tau = 5 us to the 1e-5 survival tail, production Krylov knobs)
is propagated on the GPU, written as a cell with the runner's configuration
digest and read back: the digest must match the runner's, a different
configuration must be refused, and the yield figures must agree with the
oracle's FP64 restatement of the same trajectory.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_gpu_cell_round_trip_under_resume_checks(tmp_path):
    import oracle
    import rpm_b200 as rb
    from rpm_b200 import checkpoint
    from rpm_b200 import production as p
    from rpm_b200.model import ALL_NUCLEI, FAD_NUCLEI

    nuclei = (FAD_NUCLEI[0], FAD_NUCLEI[1], ALL_NUCLEI[len(FAD_NUCLEI)])
    radicals = ("FAD", "FAD", "TrpH")
    dims = p.dimensions_for(nuclei)
    theta, sample = 90.0, 1
    h = p.build_hamiltonian(theta, 0.05, coupling=p.PRODUCTION_COUPLING, quadrupole_scale=1.0, nuclei=nuclei,
                            radicals=radicals)
    psi0 = p.random_phase_initial_state(dims, p.MASTER_SEED, sample)
    times = p.time_grid_us(p.maximum_time_us(5.0, 1e-5))
    res = p.make_propagator(h).propagate(psi0, times, rb.SingletPopulationObservable(dims))
    values = checkpoint.cell_values(times, res.observable_values, res.observable_error_bounds,
                                    res.state_error_estimates, lifetime_us=5.0, tail_bound=1e-5)
    digest = checkpoint.f14_digest(smoke=True)
    meta = {"task": {"theta_deg": theta, "scale": 1.0, "sample_id": sample}, "configuration_hash": digest,
            "stats": {"accepted_steps": res.stats.accepted_steps, "matvecs": res.stats.matvecs}}
    final = res.final_state.cpu().numpy() if hasattr(res.final_state, "cpu") else res.final_state
    path = checkpoint.write_cell(tmp_path / "cells" / "theta090_q1_s1.npz", values, final_state=final,
                                 initial_singlet=rb.singlet_population(psi0, dims), metadata=meta)
    got, got_meta = checkpoint.read_cell(path, expected_hash=digest)
    assert set(checkpoint.CELL_KEYS) <= set(got)
    assert got_meta["configuration_hash"] == digest
    with pytest.raises(ValueError, match="Incompatible checkpoint"):
        checkpoint.read_cell(path, expected_hash=checkpoint.f14_digest())
    assert got["final_state"].shape == (int(np.prod(dims)),)
    assert float(got["initial_singlet"]) == pytest.approx(1.0, abs=1e-12)
    # the same trajectory through the oracle's FP64 restatement of the reference
    href = oracle.build_hamiltonian(theta, 0.05, nuclei=nuclei, radicals=radicals, quadrupole_scale=1.0,
                                    exchange_J_uT=oracle.R2_D_PAPER_UT / -3.0, d_paper_uT=oracle.R2_D_PAPER_UT)
    ref = oracle.AdaptiveLanczosPropagator(href, minimum_dimension=24, maximum_dimension=64,
                                           state_error_budget=2.4e-5).propagate(
        psi0, times, oracle.SingletPopulationObservable(dims))
    assert abs(float(got["yield"]) - oracle.integrate_yield(times, ref.observable_values, 5.0)) < 1e-9
    assert np.max(np.abs(got["singlet_population"] - ref.observable_values)) < 1e-9
    assert float(got["quadrature_error"]) < 1e-6
