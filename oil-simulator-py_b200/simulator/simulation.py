"""``simulator.simulation`` drop-in (src/simulator/simulation.py): the IMPES
``Simulator`` with its step on the B200."""
from impes_b200.simulator import Simulator  # noqa: F401
