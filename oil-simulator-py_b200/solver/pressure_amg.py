"""``solver.pressure_amg`` drop-in (src/solver/pressure_amg.py)."""
from impes_b200.amg import _AMG_CACHE, amg_preconditioner, amg_solve  # noqa: F401
