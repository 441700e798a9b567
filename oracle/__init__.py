"""CPU oracle for the particle-fluid hot path — TEST INFRASTRUCTURE ONLY.

``sph_oracle.cpp`` restates the reference solvers (``solver/sph/solver_wcsph.py``,
``solver/sph/solver_dfsph.py``, ``solver/pbf/solver_pbf.py``) and warp-lang
1.17.0's ``wp.HashGrid`` on the CPU.  This package wraps it with ctypes.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it, and only to verify results (or as the timed
CPU baseline).  The product package never imports it.

Parity pin: the restatement is checked against golden vectors produced by
running the reference's own solver source under a substitute Warp runtime
(``tests/golden/make_golden.py``) and against the reference's known-answer
unit tests (``unit_test/unit_test_dam_break.py``).  Grid internals (cell
rounding, hash) follow warp's published algorithm and are not pinned by any
reference test.
"""

from .sph import (  # noqa: F401
    GridCfg,
    build_oracle,
    grid_build,
    grid_candidates,
    wcsph_step,
    dfsph_step,
    pbf_step,
    apic_separation,
    num_threads,
)
