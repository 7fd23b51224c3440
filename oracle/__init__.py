"""CPU oracle for the MGPCG Poisson path (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
may import this package, and only as the checker or the timed CPU baseline.
Parity against the reference itself is unpinned: the reference runs on Taichi,
which cannot be installed here.
"""
from .oracle import OracleSolver, FIELD  # noqa: F401
