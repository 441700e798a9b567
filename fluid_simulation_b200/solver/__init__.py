"""Drop-in particle-fluid solvers (module layout of the reference's ``solver`` package)."""

from .pbf import SolverPBF  # noqa: F401
from .sph.solver_dfsph import SolverDFSPH  # noqa: F401
from .sph.solver_wcsph import SolverWCSPH  # noqa: F401
