"""B200-native particle-fluid hot path (hash grid + WCSPH / DFSPH / PBF steps).

Drop-in for the solvers of SParksLz/fluid_simulation: the classes in
``fluid_simulation_b200.solver`` keep the reference's names, configs, custom
attributes and ``step(state_in, state_out, control, contacts, dt)`` contract,
and run hand-written sm_100a CUDA kernels from ``libfluid_b200.so`` through a
C ABI (``include/fluid_b200.h``).
"""

__version__ = "0.1.0"
