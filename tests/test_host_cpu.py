"""Host-side checks that need no GPU: the C ABI library, its host-built
radical-split tables, and the Python model/assembly code."""

import math
import re

import numpy as np
import pytest

import oracle
from conftest import REPO, terms_from
from rpm_b200 import _lib, model, synthetic
from rpm_b200.engine import LocalTerm, _auto_split, _DeviceSystem


def header_functions():
    text = (REPO / "include" / "rpm_b200.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(rpm_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = header_functions()
    assert len(declared) >= 15
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) - {"rpm_last_error"} <= set(_lib.SIGNATURES)
    assert lib.rpm_version() >= 1


def test_measurement_knobs_reject_unknown_values():
    # host-side setters: no device work, so they run on a machine without a GPU
    for name, bad, good in (("rpm_set_gram_kernel", 2, 1), ("rpm_set_persistent_warps", 7, 8)):
        with pytest.raises(ValueError, match="must be"):  # RPM_E_INVALID maps to ValueError
            _lib.call(name, bad)
        _lib.call(name, good)


def test_device_count_without_gpu_is_a_clean_zero_or_more():
    assert _lib.device_count() >= 0


def _dense_from_csr(ptr, col, val, n):
    out = np.zeros((n, n), dtype=complex)
    for r in range(n):
        for k in range(ptr[r], ptr[r + 1]):
            out[r, col[k]] += val[k]
    return out


@pytest.mark.parametrize("key", ["small", "prefix6", "prefix10", "full"])
def test_split_tables_match_oracle_blocks(golden, key):
    if key == "full":
        sysm = synthetic.full_system()
        dims, left, right = sysm.dimensions, sysm.left_axes, sysm.right_axes
        terms = sysm.terms(math.pi / 4, 0.0)
    else:
        dims = tuple(int(v) for v in golden[f"{key}_dims"])
        left, right = tuple(golden[f"{key}_left"]), tuple(golden[f"{key}_right"])
        terms = terms_from(golden, key, LocalTerm)
    ds = _DeviceSystem(dims, terms, left, right, host_only=True)
    assert ds.split and ds.n == math.prod(dims)
    t = ds.split_tables()
    ref = oracle.CompiledFullPairHamiltonian(dims, [oracle.LocalTerm(x.axes, x.operator) for x in terms],
                                             left_axes=left, right_axes=right)
    np.testing.assert_allclose(_dense_from_csr(t["lptr"], t["lcol"], t["lval"], ds.nl), ref.left_operator.toarray(),
                               atol=1e-13)
    np.testing.assert_allclose(_dense_from_csr(t["rptr"], t["rcol"], t["rval"], ds.nr), ref.right_operator.toarray(),
                               atol=1e-13)
    np.testing.assert_allclose(t["pair"].reshape(2, 2, 2, 2), ref.electron_pair_operator, atol=1e-14)
    # memory offsets reproduce the reference's axis permutation
    strides = np.array([math.prod(dims[a + 1:]) for a in range(len(dims))])
    grid_l = np.indices(ref.left_dimensions).reshape(len(left), -1)
    grid_r = np.indices(ref.right_dimensions).reshape(len(right), -1)
    np.testing.assert_array_equal(t["offl"], (strides[list(left)][:, None] * grid_l).sum(0))
    np.testing.assert_array_equal(t["offr"], (strides[list(right)][:, None] * grid_r).sum(0))


def test_host_only_system_rejects_bad_terms():
    sx = model.spin_operators(0.5)[0]
    with pytest.raises(ValueError, match="unique active axes"):
        _DeviceSystem((2, 2), [LocalTerm((0, 0), np.kron(sx, sx))], host_only=True)
    with pytest.raises(ValueError, match="out-of-range"):
        _DeviceSystem((2, 2), [LocalTerm((2,), sx)], host_only=True)
    with pytest.raises(ValueError, match="not Hermitian"):
        _DeviceSystem((2, 2), [LocalTerm((0,), np.array([[0, 1], [0, 0]], dtype=complex))], host_only=True)
    with pytest.raises(ValueError, match="Cross-radical"):
        _DeviceSystem((2, 2, 2), [LocalTerm((0, 2), np.kron(sx, sx))], (0,), (1, 2), host_only=True)
    with pytest.raises(ValueError, match="partition"):
        _DeviceSystem((2, 2, 2), [], (0,), (1,), host_only=True)


def test_auto_split_detection():
    sm = synthetic.small_system()
    terms = sm.terms(0.3, 0.2)
    assert _auto_split(sm.dimensions, terms) == (sm.left_axes, sm.right_axes)
    sx = model.spin_operators(0.5)[0]
    # a nuclear-nuclear coupling across radicals forbids a split
    bad = terms + [LocalTerm((2, 4), np.kron(model.spin_operators(1.0)[0], sx))]
    assert _auto_split(sm.dimensions, bad) is None


def test_model_builders_match_reference_outputs(golden):
    for s in (0.5, 1.0, 1.5):
        for name, op in zip("xyz", model.spin_operators(s)):
            np.testing.assert_allclose(op, golden[f"spin_{s}_{name}"], atol=1e-15)
    t = golden["coupling_tensor"]
    np.testing.assert_allclose(model.two_spin_coupling_operator(0.5, 1.0, t), golden["coupling_half_one"], atol=1e-14)
    np.testing.assert_allclose(model.quadrupole_operator(1.0, golden["quad_tensor"]), golden["quad_one"], atol=1e-14)
    np.testing.assert_allclose(model.efimova_hore_electron_coupling_operator(1.7, -2.3, golden["eh_axis"]),
                               golden["eh_op"], atol=1e-14)
    for key, tensor in model.QUADRUPOLE_TENSORS_MT.items():
        np.testing.assert_allclose(tensor, golden[f"qtensor_{key}"], atol=1e-15)
    for k, nuc in enumerate(model.ALL_NUCLEI):
        np.testing.assert_array_equal(nuc.tensor_mT, golden[f"hf_{k}"])


def test_production_seeds_and_states(golden):
    from rpm_b200 import production

    assert [production._seed(20260731, s) for s in range(4)] == [int(v) for v in golden["seeds"]]
    init = production.random_phase_initial_state(model.SYSTEM_DIMENSIONS, 20260731, 0)
    np.testing.assert_allclose(init[golden["init_s0_checks_idx"]], golden["init_s0_checks_val"], atol=1e-15)
    grid = production.time_grid_us(production.maximum_time_us(5.0, 1e-5))
    assert grid[-1] == pytest.approx(57.564627324851145, abs=1e-12)
    idx = production.coarse_grid_indices(grid.size)
    assert idx[0] == 0 and idx[-1] == grid.size - 1


def test_synthetic_systems_have_reference_shapes():
    full = synthetic.full_system()
    assert full.dimensions == model.SYSTEM_DIMENSIONS
    assert synthetic.small_system().dimension == 96
    assert synthetic.prefix_system(full, 3).dimension == 864
    assert synthetic.prefix_system(full, 5).dimension == 13824
    for t in full.terms(0.4, 1.3):
        np.testing.assert_allclose(t.operator, t.operator.conj().T, atol=1e-12)
    dirs = synthetic.fibonacci_sphere(12)
    assert len(dirs) == 12 and all(0 <= th <= math.pi for th, _ in dirs)


def test_batched_shape_order_groups_trajectories_by_shape():
    from types import SimpleNamespace

    from rpm_b200.batched import BatchedPropagator

    a = SimpleNamespace(dimensions=(2, 2, 3, 2), left_axes=(0, 2))
    b = SimpleNamespace(dimensions=(2, 2, 3, 2, 2), left_axes=(0, 2))
    a2 = SimpleNamespace(dimensions=(2, 2, 3, 2), left_axes=(0, 2))  # same shape as a, another system
    fake = SimpleNamespace(hamiltonians=[a, b, a2])
    assert BatchedPropagator.shape_order(fake, np.array([0, 2, 1, 1])) is None  # already one run per shape
    order = BatchedPropagator.shape_order(fake, np.array([1, 0, 1, 2, 0]))
    assert list(order) == [1, 3, 4, 0, 2]  # stable; shapes in the order of the Hamiltonian list
    grouped = np.array([1, 0, 1, 2, 0])[order]
    assert list(grouped) == [0, 2, 0, 1, 1]


@pytest.mark.parametrize("count", [4, 8, 14])
@pytest.mark.parametrize("coupling_ratio,qscale", [(None, 0.0), (-3.0, 1.0)])
def test_production_terms_match_the_oracle_builder(count, coupling_ratio, qscale):
    """The production term list (core.py:172-229) agrees with the oracle's
    restatement term by term: axes, labels, operators and radical split."""
    from rpm_b200 import production as p

    nuclei = p.selected_nuclei(count) if count < 14 else p.ALL_NUCLEI
    radicals = p.selected_radicals(count) if count < 14 else p.NUCLEAR_RADICALS
    coupling = p.UNCOUPLED if coupling_ratio is None else p.ElectronCoupling.ratio(coupling_ratio)
    dims, terms, left, right = p.production_terms(37.0, 0.05, coupling=coupling, quadrupole_scale=qscale,
                                                  nuclei=nuclei, radicals=radicals)
    ref = oracle.build_hamiltonian(37.0, 0.05, nuclei=nuclei, radicals=radicals, quadrupole_scale=qscale,
                                   exchange_J_uT=coupling.exchange_J_uT, d_paper_uT=coupling.d_paper_uT,
                                   dipolar_axis=coupling.dipolar_axis)
    assert tuple(dims) == tuple(ref.dimensions)
    assert (tuple(left), tuple(right)) == (tuple(ref.left_axes), tuple(ref.right_axes))
    assert [t.label for t in terms] == [t.label for t in ref.terms]
    for t, r in zip(terms, ref.terms):
        assert tuple(t.axes) == tuple(r.axes)
        np.testing.assert_allclose(t.operator, r.operator, rtol=0, atol=1e-12)


def test_production_terms_error_texts():
    from rpm_b200 import production as p

    n0, n1 = p.ALL_NUCLEI[0], p.ALL_NUCLEI[1]
    with pytest.raises(ValueError, match="same length"):
        p.production_terms(0.0, 0.05, nuclei=(n0,), radicals=("FAD", "TrpH"))
    with pytest.raises(ValueError, match="duplicate radical/name keys"):
        p.production_terms(0.0, 0.05, nuclei=(n0, n0), radicals=("FAD", "FAD"))
    with pytest.raises(ValueError, match="belong to FAD or TrpH"):
        p.production_terms(0.0, 0.05, nuclei=(n0, n1), radicals=("FAD", "Flavin"))


def test_population_bounds_match_the_scalar_rule():
    from rpm_b200.engine import population_bounds, state_error_to_population_bound

    rng = np.random.default_rng(3)
    se = np.concatenate([rng.uniform(-1e-3, 1e-3, 2000), rng.uniform(0.0, 2.0, 200), [0.0, -0.0, 1e-300, np.inf]])
    want = np.array([state_error_to_population_bound(v) for v in se])
    np.testing.assert_array_equal(population_bounds(se.reshape(-1, 4)), want.reshape(-1, 4))


def test_oracle_linear_algebra_rejects_bad_sizes_before_any_launch():
    import ctypes

    size = ctypes.c_longlong()
    _lib.call("rpm_he_eigh_workspace", 576, 3, ctypes.byref(size))
    n, nn = 576, 576 * 576
    assert size.value >= 3 * (5 * n * 8 + 8 + nn * 24)
    for bad in ((1, 1), (2000, 1), (8, 0)):
        with pytest.raises(ValueError):
            _lib.call("rpm_he_eigh_workspace", bad[0], bad[1], ctypes.byref(size))
    null = ctypes.c_void_p()
    with pytest.raises(ValueError):  # not a power of two
        _lib.call("rpm_fft_pow2", 6, 1, null, null, 0, null)
    with pytest.raises(ValueError):
        _lib.call("rpm_zgemm_hn", 0, 1, null, null, null, null)
    with pytest.raises(ValueError):
        _lib.call("rpm_spectrum_mac", ctypes.c_longlong(0), null, null, null, null)
