"""``simulator.fluid`` drop-in (src/simulator/fluid.py)."""
from impes_b200.simulator import Fluid  # noqa: F401
