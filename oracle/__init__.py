"""CPU oracle for the radical-pair hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the ``rpm_b200`` package imports this
package.  It is imported by ``tests/``, by ``__graft_entry__.smoke()`` (as the
checker of one small GPU run) and by ``bench.py``'s CPU-baseline leg and its
``--impl reference`` arm.  It is never the thing measured for the GPU path and
never a fallback for it.

The oracle is a NumPy restatement of the reference's FP64 algorithm
(``Realistic system size/code/rpm_statevector_engine.py`` and friends, cited
per function).  It is pinned against fixtures that were produced by running
the reference itself (``tests/golden/make_golden.py``) and against the
reference's own known-answer tests.
"""

from .rpm_oracle import *  # noqa: F401,F403
