"""Checkpoint cells: atomic write, keys, hash check (host only)."""

import json

import numpy as np
import pytest

from rpm_b200 import checkpoint


def _values():
    t = np.arange(5) * 0.1
    return {"yield": np.array(0.27), "coarse_yield": np.array(0.27), "quadrature_error": np.array(1e-9),
            "yield_propagation_estimate": np.array(1e-7), "yield_tail_bound": np.array(1e-5), "times_us": t,
            "singlet_population": np.full(5, 0.5), "population_error_estimate": np.zeros(5),
            "state_error_estimates": np.zeros(5)}


def test_cell_roundtrip_and_hash(tmp_path):
    cfg = {"seed": 20260731, "krylov": [24, 64]}
    h = checkpoint.configuration_hash(cfg)
    path = checkpoint.write_cell(tmp_path / "cells" / "Q0_th000.000_s000.npz", _values(), final_state=np.ones(8),
                                 initial_singlet=1.0, metadata={"configuration_hash": h, "task": {"sample_id": 0}})
    assert path.exists() and not list(path.parent.glob("*.tmp"))
    values, meta = checkpoint.read_cell(path, expected_hash=h)
    assert set(checkpoint.CELL_KEYS) <= set(values)
    assert meta["task"]["sample_id"] == 0
    with pytest.raises(ValueError, match="Incompatible"):
        checkpoint.read_cell(path, expected_hash="0" * 64)


def test_cell_rejects_missing_keys_and_nonfinite(tmp_path):
    v = _values()
    del v["yield"]
    with pytest.raises(ValueError):
        checkpoint.write_cell(tmp_path / "a.npz", v, final_state=np.ones(2), initial_singlet=1.0, metadata={})
    v = _values()
    v["yield"] = np.array(np.nan)
    p = checkpoint.write_cell(tmp_path / "b.npz", v, final_state=np.ones(2), initial_singlet=1.0, metadata={})
    with pytest.raises(ValueError, match="Nonfinite"):
        checkpoint.read_cell(p)
    assert json.loads(str(np.load(p)["metadata_json"])) == {}


def test_f14_digest_matches_the_reference_runner():
    """configuration_hash of the full-size runner's cells, pinned to digests
    that the reference's own Config(...).digest produced
    (tests/golden/make_checkpoint_golden.py)."""
    from conftest import GOLDEN

    cases = json.loads((GOLDEN / "f14_digests.json").read_text())
    assert len(cases) >= 4
    for case in cases:
        mine = json.loads(json.dumps(checkpoint.f14_stable_dict(**case["config"]), sort_keys=True))
        assert mine == case["stable_dict"]
        assert checkpoint.f14_digest(**case["config"]) == case["digest"]
