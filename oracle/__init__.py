"""CPU oracle for the IMPES hot path (test infrastructure only).

This package is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` may import it.  It restates, in float64 numpy/scipy, the
reference's algorithm for the IMPES time step of researchim-ai/oil-simulator-py:

* ``oracle.impes`` -- pressure assembly and explicit saturation update
  (``src/simulator/simulation.py``, ``fluid.py``, ``pvt.py``, ``well.py``),
* ``oracle.amg``   -- the Ruge--Stueben ``ClassicalAMG`` hierarchy, V-cycle and
  ``amg_solve`` (``src/solver/classical_amg.py``, ``pressure_amg.py``).

Every function cites the reference file:line it follows.  Parity of this
restatement is pinned against the reference itself (imported in the build
container) through the golden fixtures in ``tests/golden/`` and the script that
made them, ``tests/golden/make_golden.py``.
"""
