"""``simulator.well`` drop-in (src/simulator/well.py)."""
from impes_b200.simulator import Well, WellManager  # noqa: F401
