"""Golden configuration digests of the reference's full-size runner.

Run once with the reference next to the checkout:

    python tests/golden/make_checkpoint_golden.py <RPM checkout>

It imports ``rpm_full14_quadrupole_experiment`` from the reference (through
``make_golden.load_reference``, which stubs matplotlib) and writes
``f14_digests.json``: the ``Config(...).digest`` of a few configurations (the
``configuration_hash`` its cells carry and its resume checks) and their
``stable_dict()`` records.
"""

from __future__ import annotations

import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

from make_golden import load_reference  # noqa: E402

CASES = [{}, {"smoke": True}, {"smoke": True, "seed": 5, "samples": 2, "state_error_budget": 1e-7},
         {"lifetime_us": 1.0, "tail_bound": 1e-4}]


def main(root: Path) -> None:
    load_reference(root)
    import rpm_full14_quadrupole_experiment as F14  # noqa: N812

    out = []
    for kw in CASES:
        cfg = F14.Config(**kw)
        out.append({"config": kw, "digest": cfg.digest,
                    "stable_dict": json.loads(json.dumps(cfg.stable_dict(), sort_keys=True))})
    (HERE / "f14_digests.json").write_text(json.dumps(out, indent=1) + "\n")
    print([c["digest"][:12] for c in out])


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(f"usage: python {Path(__file__).name} <path of the RPM checkout>")
    main(Path(sys.argv[1]))
