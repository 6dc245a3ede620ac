"""Unequal Haberkorn recombination rates on the batched path (Arnoldi) against a dense oracle.

There is no reference implementation of kS != kT (the reference propagates
with equal rates only), so the oracle is a dense restatement: the state is
propagated exactly under H - (i/2)(kS P_S + kT P_T).  Bars: populations of
the factored state within 1e-5 and yields within 1e-6 (the batched path's
complex64 contract); H psi within 1e-12 (complex128) / 2e-6 (complex64).
"""

import math

import numpy as np
import pytest

import oracle


def _small(rb, seed=31):
    from rpm_b200 import synthetic

    sysm = synthetic.make_system(seed, (1, 3), (0, 3))  # 768 dimensions, shape-specialised passes
    terms = sysm.terms(0.7, 0.4)
    h = rb.CompiledFullPairHamiltonian(sysm.dimensions, terms, left_axes=sysm.left_axes, right_axes=sysm.right_axes)
    dense = oracle.MatrixFreeHamiltonian(sysm.dimensions, [oracle.LocalTerm(t.axes, t.operator) for t in terms]).explicit_matrix()
    return sysm, h, dense


def test_dense_oracle_equal_rates_match_hermitian_oracle():
    from rpm_b200 import synthetic

    sysm = synthetic.small_system()
    terms = sysm.terms(0.3, 0.0)
    ho = oracle.MatrixFreeHamiltonian(sysm.dimensions, [oracle.LocalTerm(t.axes, t.operator) for t in terms])
    psi = synthetic.random_phase_vectors(sysm.dimensions, 1, 4)[0]
    times = np.arange(401) * 0.0025
    factored, y = oracle.haberkorn_dense(ho.explicit_matrix(), sysm.dimensions, psi, times, 1.0, 1.0)
    w, v = np.linalg.eigh(ho.explicit_matrix())
    c = v.conj().T @ psi
    pops = np.array([oracle.singlet_population(v @ (np.exp(-1j * w * t) * c), sysm.dimensions) for t in times])
    np.testing.assert_allclose(factored, pops, atol=1e-12)
    assert y == pytest.approx(oracle.integrate_yield(times, pops, 1.0), abs=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("rates", [(1.0, 2.0), (2.0, 1.0)])
def test_unequal_rates_match_dense_oracle(rates):
    import rpm_b200 as rb
    from rpm_b200 import synthetic
    from rpm_b200.batched import BatchedPropagator

    sysm, h, dense = _small(rb)
    assert h._system.fast_hpsi
    h.set_recombination_rates(*rates)
    assert h.recombination_rates == rates
    psi = synthetic.random_phase_vectors(sysm.dimensions, 3, 17)
    times = np.arange(801) * 0.00125  # 0 .. 1 us
    bp = BatchedPropagator([h], krylov_dimension=24, state_error_budget=1e-9)
    out = bp.propagate(list(psi), times, system_index=[0, 0, 0])
    for b in range(3):
        factored, y = oracle.haberkorn_dense(dense, sysm.dimensions, psi[b], times, *rates)
        assert np.max(np.abs(out.observable_values[b] - factored)) < 1e-5
        assert abs(out.yields[b] - y) < 1e-6
    from rpm_b200._lib import RpmError

    with pytest.raises(RpmError):
        rb.AdaptiveLanczosPropagator(h).propagate(psi[0], times[:11], rb.SingletPopulationObservable(sysm.dimensions))


@pytest.mark.gpu
def test_non_hermitian_action_matches_dense():
    import torch

    import rpm_b200 as rb

    sysm, h, dense = _small(rb)
    ks, kt = 0.5, 3.0
    h.set_recombination_rates(ks, kt)
    m = math.prod(sysm.dimensions) // 4
    ps4 = np.zeros((4, 4), dtype=complex)
    ps4[1, 1] = ps4[2, 2] = 0.5
    ps4[1, 2] = ps4[2, 1] = -0.5
    pt = np.kron(np.eye(4) - ps4, np.eye(m))
    expected_op = dense - 0.5j * (kt - ks) * pt  # common decay exp(-ks t / 2) factored out
    v = np.random.default_rng(2).normal(size=dense.shape[0]) + 1j * np.random.default_rng(3).normal(size=dense.shape[0])
    ref = expected_op @ v
    got = h.matvec(v)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-12
    x = torch.from_numpy(v).to("cuda", torch.complex64)
    y = torch.empty_like(x)
    h.apply(x, y, precision=64)
    assert np.linalg.norm(y.cpu().numpy() - ref) / np.linalg.norm(ref) < 2e-6


@pytest.mark.gpu
def test_arnoldi_full_size_near_equal_rates_match_lanczos():
    """Arnoldi at 221,184 dimensions: rates (1, 1 + 1e-9) against the Hermitian Lanczos path at tau = 1 us."""
    import rpm_b200 as rb
    from rpm_b200 import synthetic
    from rpm_b200.batched import BatchedPropagator

    full = synthetic.full_system()
    terms = full.terms(math.pi / 4, 0.0)
    mk = lambda: rb.CompiledFullPairHamiltonian(full.dimensions, terms, left_axes=full.left_axes,
                                                right_axes=full.right_axes)
    h_arn, h_lan = mk(), mk()
    h_arn.set_recombination_rates(1.0, 1.0 + 1e-9)
    assert h_arn._system.recombination()[2]  # non-Hermitian: Arnoldi
    psi = synthetic.random_phase_vectors(full.dimensions, 2, 44)
    times = np.arange(161) * 0.00125  # 0 .. 0.2 us
    a = BatchedPropagator([h_arn], krylov_dimension=32, state_error_budget=1e-8).propagate(list(psi), times,
                                                                                          system_index=[0, 0])
    l = BatchedPropagator([h_lan], krylov_dimension=32, state_error_budget=1e-8).propagate(list(psi), times,
                                                                                          system_index=[0, 0],
                                                                                          lifetime_us=1.0)
    assert np.max(np.abs(a.observable_values - l.observable_values)) < 1e-5
    assert np.max(np.abs(a.yields - l.yields)) < 1e-6


@pytest.mark.gpu
def test_non_hermitian_action_on_the_general_cube_kernels():
    """A layout without shape-specialised passes (96 dimensions): complex128 and complex64 H psi."""
    import torch

    import rpm_b200 as rb
    from rpm_b200 import synthetic

    sysm = synthetic.small_system()
    terms = sysm.terms(0.4, 1.1)
    h = rb.CompiledFullPairHamiltonian(sysm.dimensions, terms, left_axes=sysm.left_axes, right_axes=sysm.right_axes)
    assert not h._system.fast_hpsi
    dense = oracle.MatrixFreeHamiltonian(sysm.dimensions, [oracle.LocalTerm(t.axes, t.operator) for t in terms]).explicit_matrix()
    ks, kt = 1.0, 2.0
    h.set_recombination_rates(ks, kt)
    m = math.prod(sysm.dimensions) // 4
    ps4 = np.zeros((4, 4), dtype=complex)
    ps4[1, 1] = ps4[2, 2] = 0.5
    ps4[1, 2] = ps4[2, 1] = -0.5
    expected_op = dense - 0.5j * (kt - ks) * np.kron(np.eye(4) - ps4, np.eye(m))
    rng = np.random.default_rng(8)
    v = rng.normal(size=dense.shape[0]) + 1j * rng.normal(size=dense.shape[0])
    ref = expected_op @ v
    assert np.linalg.norm(h.matvec(v) - ref) / np.linalg.norm(ref) < 1e-12
    x = torch.from_numpy(v).to("cuda", torch.complex64)
    y = torch.empty_like(x)
    h.apply(x, y, precision=64)
    assert np.linalg.norm(y.cpu().numpy() - ref) / np.linalg.norm(ref) < 2e-6


@pytest.mark.gpu
def test_uneven_sizes_with_unequal_rates_match_dense_oracle():
    """Uneven system sizes (96, 768 and 864 dimensions, interleaved) with kS = 1e6, kT = 2e6 s^-1 in one
    propagate call: one launch group per shape (fused Arnoldi passes for the 768-dimension shape, the
    general cube kernels for the others)."""
    import rpm_b200 as rb
    from rpm_b200 import synthetic
    from rpm_b200.batched import BatchedPropagator

    systems = [synthetic.small_system(), synthetic.make_system(31, (1, 3), (0, 3)),
               synthetic.prefix_system(synthetic.full_system(), 3)]
    rates = (1.0, 2.0)
    hams, dense = [], []
    for k, sysm in enumerate(systems):
        terms = sysm.terms(0.3 + 0.4 * k, 0.2 * k)
        h = rb.CompiledFullPairHamiltonian(sysm.dimensions, terms, left_axes=sysm.left_axes,
                                           right_axes=sysm.right_axes)
        h.set_recombination_rates(*rates)
        hams.append(h)
        dense.append(oracle.MatrixFreeHamiltonian(sysm.dimensions, [oracle.LocalTerm(t.axes, t.operator)
                                                                   for t in terms]).explicit_matrix())
    assert [h._system.fast_hpsi for h in hams] == [False, True, False]
    index = [0, 1, 2, 0, 1, 2]
    states = [synthetic.random_phase_vectors(systems[k].dimensions, 1, 50 + b)[0] for b, k in enumerate(index)]
    times = np.arange(801) * 0.00125  # 0 .. 1 us
    bp = BatchedPropagator(hams, krylov_dimension=24, state_error_budget=1e-9)
    assert bp.shape_order(np.array(index)) is not None
    out = bp.propagate(states, times, system_index=index)
    for b, (psi, k) in enumerate(zip(states, index)):
        factored, y = oracle.haberkorn_dense(dense[k], systems[k].dimensions, psi, times, *rates)
        assert np.max(np.abs(out.observable_values[b] - factored)) < 1e-5
        assert abs(out.yields[b] - y) < 1e-6
