"""B200-native IMPES pressure/saturation path (researchim-ai/oil-simulator-py drop-in).

Importing ``impes_b200`` itself is light (scenario inputs only); the compute
modules (``impes_b200.amg``, ``impes_b200.simulator``) load
``libimpes_b200.so`` and raise ImportError if it is missing.
"""
__all__ = ["scenarios"]
