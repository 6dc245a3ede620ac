"""Device-driven plain propagation (rpm_plain_propagate) against the host-driven loop.

With the singlet population observable the plain FP64 propagator decides
every Krylov step on the device (candidate spectra, embedded errors, the
first dimension within the budget, observation points, the new state) and
reads one record per step.  The reference controller's decisions
(rpm_statevector_engine.py:717-933) must be unchanged: the same accepted and
rejected steps, H psi count and largest dimension as the host-driven loop,
populations within 1e-12, the final state within 1e-11 and the accumulated
state-error estimates within 1e-3 relative (they are differences of nearly
equal coefficient vectors, near the roundoff floor at tight budgets).
"""

import math

import numpy as np
import pytest

from conftest import terms_from

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rb():
    import rpm_b200

    return rpm_b200


def _both(rb, h, psi, times, dims, **knobs):
    out = []
    for device in (False, True):
        prop = rb.AdaptiveLanczosPropagator(h, device_steps=device, **knobs)
        out.append(prop.propagate(psi, times, rb.SingletPopulationObservable(dims)))
    return out


def _same(host, dev):
    hs, ds = host.stats, dev.stats
    assert (ds.accepted_steps, ds.rejected_steps, ds.matvecs, ds.maximum_krylov_dimension) == \
        (hs.accepted_steps, hs.rejected_steps, hs.matvecs, hs.maximum_krylov_dimension)
    assert ds.minimum_step_us == pytest.approx(hs.minimum_step_us, rel=1e-12)
    assert ds.maximum_step_us == pytest.approx(hs.maximum_step_us, rel=1e-12)
    # error estimates are differences of nearly equal coefficient vectors: the eigen-solvers'
    # rounding moves them in the fifth digit near the roundoff floor
    assert ds.accumulated_state_error == pytest.approx(hs.accumulated_state_error, rel=1e-3, abs=1e-20)
    np.testing.assert_allclose(dev.observable_values, host.observable_values, atol=1e-12)
    np.testing.assert_allclose(dev.state_error_estimates, host.state_error_estimates, rtol=1e-3, atol=1e-20)
    np.testing.assert_allclose(dev.observable_error_bounds, host.observable_error_bounds, rtol=1e-3, atol=1e-20)
    np.testing.assert_allclose(dev.final_state, host.final_state, atol=1e-11)
    assert ds.maximum_norm_error == pytest.approx(hs.maximum_norm_error, abs=1e-13)


@pytest.mark.parametrize("key", ["small", "prefix6", "prefix10"])
@pytest.mark.parametrize("knobs", [dict(minimum_dimension=8, maximum_dimension=40, state_error_budget=1e-10),
                                   dict(minimum_dimension=24, maximum_dimension=64),
                                   dict(minimum_dimension=8, maximum_dimension=16, state_error_budget=1e-11)])
def test_device_steps_match_host_loop(rb, golden, key, knobs):
    dims = tuple(int(v) for v in golden[f"{key}_dims"])
    h = rb.CompiledFullPairHamiltonian(dims, terms_from(golden, key, rb.LocalTerm),
                                       left_axes=tuple(golden[f"{key}_left"]), right_axes=tuple(golden[f"{key}_right"]))
    psi = golden[f"{key}_psi0"]
    psi = psi[0] if psi.ndim == 2 else psi
    times = golden[f"{key}_times"]
    host, dev = _both(rb, h, psi, times, dims, **knobs)
    _same(host, dev)


def test_device_steps_with_rejections_and_exact_bases(rb):
    """An 8-dimensional system: every basis is exact (8 < the minimum 12), and a 2-us first step
    forces rejections on the 3..6 ladder."""
    sx, sy, sz = rb.spin_operators(0.5)
    terms = (rb.LocalTerm((0,), 0.7 * sx + 0.2 * sz), rb.LocalTerm((1, 2), 0.4 * np.kron(sy, sx) + 0.3 * np.kron(sz, sz)))
    h = rb.MatrixFreeHamiltonian((2, 2, 2), terms)
    psi = rb.singlet_initial_state((2, 2, 2), np.random.default_rng(6))
    times = np.linspace(0.0, 3.0, 31)
    for knobs in (dict(minimum_dimension=12, maximum_dimension=16),
                  dict(minimum_dimension=3, maximum_dimension=6, dimension_increment=1, embedded_offset=2,
                       state_error_budget=1e-9, initial_step_us=2.0, maximum_step_us=2.0)):
        host, dev = _both(rb, h, psi, times, (2, 2, 2), **knobs)
        _same(host, dev)
    assert host.stats.rejected_steps > 0


def test_device_steps_full_size(rb):
    from rpm_b200 import synthetic

    full = synthetic.full_system()
    h = rb.CompiledFullPairHamiltonian(full.dimensions, full.terms(math.pi / 4, 0.0), left_axes=full.left_axes,
                                       right_axes=full.right_axes)
    psi = synthetic.random_phase_vectors(full.dimensions, 1, 7)[0]
    times = np.arange(41) * 0.00125
    host, dev = _both(rb, h, psi, times, full.dimensions, minimum_dimension=8, maximum_dimension=40,
                      state_error_budget=1e-10)
    _same(host, dev)


def test_device_steps_minimum_step_error(rb, golden):
    key = "small"
    dims = tuple(int(v) for v in golden[f"{key}_dims"])
    h = rb.CompiledFullPairHamiltonian(dims, terms_from(golden, key, rb.LocalTerm),
                                       left_axes=tuple(golden[f"{key}_left"]), right_axes=tuple(golden[f"{key}_right"]))
    prop = rb.AdaptiveLanczosPropagator(h, minimum_dimension=6, maximum_dimension=8, state_error_budget=1e-14,
                                        minimum_step_us=0.01)
    with pytest.raises(RuntimeError, match="fell below the configured minimum"):
        prop.propagate(golden[f"{key}_psi0"][0], golden[f"{key}_times"], rb.SingletPopulationObservable(dims))
