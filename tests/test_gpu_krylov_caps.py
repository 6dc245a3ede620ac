"""Per-system Krylov dimensions in one batch (rpm_batch_set_krylov_caps).

A trajectory whose system has cap c ends its Krylov basis after c
iterations, so uneven system sizes in one launch each run at their own
dimension.  Bars as for the batched path: populations within 1e-5 and yields
within 1e-6 of the FP64 path (Lanczos) or of the dense oracle (Arnoldi, with
unequal recombination rates); every accepted step of a capped trajectory
costs exactly c H psi products, and the stats report c as its dimension.
"""

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

YIELD_TOL = 1e-6
POP_TOL = 1e-5


def _ham(rb, sysm, th, ph):
    return rb.CompiledFullPairHamiltonian(sysm.dimensions, sysm.terms(th, ph), left_axes=sysm.left_axes,
                                          right_axes=sysm.right_axes)


@pytest.mark.parametrize("kernel,reorth", [("persistent", 0), ("passes", 0), ("persistent", 5)])
def test_caps_per_system_match_fp64(kernel, reorth):
    import rpm_b200 as rb
    from rpm_b200 import synthetic
    from rpm_b200.batched import BatchedPropagator

    full = synthetic.full_system()
    systems = [synthetic.prefix_system(full, 3), synthetic.prefix_system(full, 5)]  # 864 and 13,824 dimensions
    hams = [_ham(rb, systems[0], 0.4, 0.3), _ham(rb, systems[1], 1.1, 2.0)]
    caps = [12, 20]
    index = [0, 1, 1, 0, 1]
    states = [synthetic.random_phase_vectors(systems[k].dimensions, 1, 70 + b)[0] for b, k in enumerate(index)]
    times = np.arange(241) * 0.00125  # 0 .. 0.3 us
    bp = BatchedPropagator(hams, krylov_dimension=32, state_error_budget=1e-9, krylov_caps=caps,
                           lanczos_kernel=kernel, reorth_period=reorth)
    out = bp.propagate(states, times, system_index=index, lifetime_us=1.0)
    assert not out.status.any()
    for b, k in enumerate(index):
        ref = rb.AdaptiveLanczosPropagator(hams[k], minimum_dimension=8, maximum_dimension=40,
                                           state_error_budget=1e-10).propagate(
            states[b], times, rb.SingletPopulationObservable(systems[k].dimensions)).observable_values
        assert np.max(np.abs(out.observable_values[b] - ref)) < POP_TOL
        assert abs(out.yields[b] - rb.integrate_yield(times, ref, 1.0)) < YIELD_TOL
        s = out.stats[b]
        assert s.maximum_krylov_dimension == caps[k]
        assert s.matvecs == s.accepted_steps * caps[k]
    # a capped system steps exactly as a batch of that dimension alone
    alone = BatchedPropagator([hams[0]], krylov_dimension=caps[0], state_error_budget=1e-9, lanczos_kernel=kernel,
                              reorth_period=reorth)
    first = [b for b, k in enumerate(index) if k == 0]
    solo = alone.propagate([states[b] for b in first], times, system_index=[0] * len(first), lifetime_us=1.0)
    for i, b in enumerate(first):
        assert solo.stats[i].accepted_steps == out.stats[b].accepted_steps
        assert abs(solo.yields[i] - out.yields[b]) < 1e-9


def test_caps_with_unequal_rates_match_dense_oracle():
    """Arnoldi (kS = 1e6, kT = 2e6 s^-1) on 96-, 768- and 864-dimension systems with caps 16, 0 (the
    batch's 24) and 20.  (The Arnoldi controller steps by whole observation spacings, so a cap must
    meet the budget over one spacing: dimension 10 does not at a 1e-9 budget.)"""
    import rpm_b200 as rb
    from rpm_b200 import synthetic
    from rpm_b200.batched import BatchedPropagator

    systems = [synthetic.small_system(), synthetic.make_system(31, (1, 3), (0, 3)),
               synthetic.prefix_system(synthetic.full_system(), 3)]
    rates = (1.0, 2.0)
    caps = [16, 0, 20]
    hams, dense = [], []
    for k, sysm in enumerate(systems):
        terms = sysm.terms(0.3 + 0.4 * k, 0.2 * k)
        h = rb.CompiledFullPairHamiltonian(sysm.dimensions, terms, left_axes=sysm.left_axes,
                                           right_axes=sysm.right_axes)
        h.set_recombination_rates(*rates)
        hams.append(h)
        dense.append(oracle.MatrixFreeHamiltonian(sysm.dimensions, [oracle.LocalTerm(t.axes, t.operator)
                                                                   for t in terms]).explicit_matrix())
    index = [0, 1, 2, 2, 1, 0]
    states = [synthetic.random_phase_vectors(systems[k].dimensions, 1, 60 + b)[0] for b, k in enumerate(index)]
    times = np.arange(801) * 0.00125  # 0 .. 1 us
    out = BatchedPropagator(hams, krylov_dimension=24, state_error_budget=1e-9, krylov_caps=caps).propagate(
        states, times, system_index=index)
    for b, (psi, k) in enumerate(zip(states, index)):
        factored, y = oracle.haberkorn_dense(dense[k], systems[k].dimensions, psi, times, *rates)
        assert np.max(np.abs(out.observable_values[b] - factored)) < POP_TOL
        assert abs(out.yields[b] - y) < YIELD_TOL
        cap = caps[k] or 24
        assert out.stats[b].maximum_krylov_dimension == cap
        assert out.stats[b].matvecs == out.stats[b].accepted_steps * cap


def test_invalid_caps_are_refused():
    import rpm_b200 as rb
    from rpm_b200 import synthetic
    from rpm_b200._lib import RpmError
    from rpm_b200.batched import BatchedPropagator

    sysm = synthetic.prefix_system(synthetic.full_system(), 3)
    hams = [_ham(rb, sysm, 0.2, 0.0), _ham(rb, sysm, 0.9, 1.0)]
    for caps in ([1, 8], [8, 33], [8, 8, 8]):
        with pytest.raises((RpmError, ValueError)):
            BatchedPropagator(hams, krylov_dimension=32, krylov_caps=caps)
    BatchedPropagator(hams, krylov_dimension=32, krylov_caps=[0, 32])
