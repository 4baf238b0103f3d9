"""CPU oracle for the RBF-PUM transfer (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package.  The product (``pacman_b200``) never
loads it.
"""
from .oracle import (  # noqa: F401
    OraclePlan,
    build,
    ensure_built,
    fe_nearest,
    interpolate,
    mls_interpolate,
    set_threads,
    wendland,
)
