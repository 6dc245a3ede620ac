"""Tensor-core singlet Gram (k_b_gram_tc) against the CUDA-core kernel (GPU).

The Gram only feeds the populations at the observation points: the states,
steps and Krylov bases of a batched propagation are the same with either
kernel, so the populations must agree to the Gram's rounding.  The tensor
cores' FP32 accumulation rounds towards zero; with the TF32 high/low split and
the large term drained after every 32-row chunk (four accumulating MMAs) the
Gram carries a relative error of about 1.5e-7 (measured against the CUDA-core
kernel: 1.1e-7 on populations of order 0.3).  The bar here is 3e-7 on the
populations, and the yields against the FP64 plain path stay within the
batched path's 1e-6 bar.  The reference forms this projection per
basis in rpm_statevector_engine.py:521-529.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

POP_AGREE = 3e-7


@pytest.fixture(scope="module")
def rb():
    import rpm_b200

    return rpm_b200


def _both(rb, hams, states, times, sys_idx, **knobs):
    from rpm_b200 import _lib
    from rpm_b200.batched import BatchedPropagator

    out = []
    try:
        for kernel in (0, 1):
            _lib.call("rpm_set_gram_kernel", kernel)
            bp = BatchedPropagator(hams, **knobs)
            out.append(bp.propagate(list(states), times, system_index=sys_idx, lifetime_us=1.0))
    finally:
        _lib.call("rpm_set_gram_kernel", 1)
    return out


def test_full_system_populations_match_cuda_core_gram(rb):
    from rpm_b200 import synthetic

    full = synthetic.full_system()
    dirs = synthetic.fibonacci_sphere(2)
    hams = [rb.CompiledFullPairHamiltonian(full.dimensions, full.terms(th, ph), left_axes=full.left_axes,
                                           right_axes=full.right_axes) for th, ph in dirs]
    states = synthetic.random_phase_vectors(full.dimensions, 4, 11)
    times = np.arange(41) * 0.00125
    sys_idx = np.array([0, 0, 1, 1], dtype=np.int32)
    cuda_core, tensor = _both(rb, hams, states, times, sys_idx, krylov_dimension=40, state_error_budget=5e-7)
    assert [s.accepted_steps for s in cuda_core.stats] == [s.accepted_steps for s in tensor.stats]
    np.testing.assert_allclose(tensor.observable_values, cuda_core.observable_values, rtol=0, atol=POP_AGREE)
    np.testing.assert_allclose(tensor.yields, cuda_core.yields, rtol=0, atol=POP_AGREE)


def test_uneven_sizes_and_short_bases(rb):
    """Three system sizes in one batch (row ranges that end inside a chunk,
    blocks without rows) and a small Krylov dimension (most operand rows zero)."""
    from rpm_b200 import synthetic

    full = synthetic.full_system()
    hams, dims = [], []
    for per, (th, ph) in ((3, (0.3, 0.0)), (5, (1.2, 2.0)), (14, (0.7, 1.1))):
        sub = synthetic.prefix_system(full, per) if per < 14 else full
        dims.append(sub.dimensions)
        hams.append(rb.CompiledFullPairHamiltonian(sub.dimensions, sub.terms(th, ph), left_axes=sub.left_axes,
                                                   right_axes=sub.right_axes))
    states = []
    for k, d in enumerate(dims):
        states.extend(synthetic.random_phase_vectors(d, 2, 20 + k))
    sys_idx = np.repeat(np.arange(3, dtype=np.int32), 2)
    times = np.arange(41) * 0.00125
    for m in (8, 24):
        cuda_core, tensor = _both(rb, hams, states, times, sys_idx, krylov_dimension=m, state_error_budget=1e-7)
        np.testing.assert_allclose(tensor.observable_values, cuda_core.observable_values, rtol=0, atol=POP_AGREE)


def test_tensor_core_yields_within_the_fp64_bar(rb):
    from rpm_b200 import synthetic
    from rpm_b200.batched import BatchedPropagator

    full = synthetic.full_system()
    sub = synthetic.prefix_system(full, 10)
    h = rb.CompiledFullPairHamiltonian(sub.dimensions, sub.terms(0.9, 0.4), left_axes=sub.left_axes,
                                       right_axes=sub.right_axes)
    states = synthetic.random_phase_vectors(sub.dimensions, 2, 5)
    times = np.arange(401) * 0.00125
    out = BatchedPropagator([h], krylov_dimension=32, state_error_budget=1e-9).propagate(list(states), times,
                                                                                          lifetime_us=1.0)
    for b in range(2):
        ref = rb.AdaptiveLanczosPropagator(h, minimum_dimension=8, maximum_dimension=40,
                                           state_error_budget=1e-10).propagate(
            states[b], times, rb.SingletPopulationObservable(sub.dimensions))
        y = rb.integrate_yield(times, ref.observable_values, 1.0)
        assert abs(out.yields[b] - y) < 1e-6
