"""TEST INFRASTRUCTURE ONLY: the CPU checker of the FASOLT3 hot path.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this package.  See ``fasolt_oracle.h`` for what it restates
and for its parity status.
"""
from .oracle import OracleSolver, build, LIB_PATH  # noqa: F401
