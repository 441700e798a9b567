from .solver_pbf import SolverPBF  # noqa: F401
