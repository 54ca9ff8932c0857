"""CPU oracle for deconlib's 3D deconvolution path (RL and Hessian PDHG).

TEST INFRASTRUCTURE ONLY.  This package is the checker the CUDA product is
compared against.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` may import it; ``deconlib_b200`` never does.

Parity pin: ``tests/test_oracle_golden.py`` checks it against golden vectors
generated from the reference's own source by ``tests/golden/make_golden.py``.
"""

from . import ops, solvers  # noqa: F401
