"""``simulator.pvt`` drop-in (src/simulator/pvt.py)."""
from impes_b200.simulator import PVTTable  # noqa: F401
