import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))

GOLDEN = REPO / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and librpm_b200.so")


@pytest.fixture(scope="session")
def golden():
    with np.load(GOLDEN / "reference_golden.npz") as data:
        return {k: data[k] for k in data.files}


def terms_from(golden, prefix, term_cls):
    """Rebuild a term list stored by tests/golden/make_golden.py."""
    axes, sizes, ops = golden[f"{prefix}_axes"], golden[f"{prefix}_sizes"], golden[f"{prefix}_ops"]
    out, pos = [], 0
    for k in range(len(sizes)):
        d = int(sizes[k])
        op = ops[pos:pos + d * d].reshape(d, d)
        pos += d * d
        out.append(term_cls(tuple(int(a) for a in axes[k] if a >= 0), op, f"term{k}"))
    return out


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
