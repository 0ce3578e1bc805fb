"""``simulator.reservoir`` drop-in (src/simulator/reservoir.py)."""
from impes_b200.simulator import Reservoir  # noqa: F401
