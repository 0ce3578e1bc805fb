"""``solver.classical_amg`` drop-in (src/solver/classical_amg.py)."""
from impes_b200.amg import ClassicalAMG, _apply_reference_fix  # noqa: F401
