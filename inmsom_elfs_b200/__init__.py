"""B200-native barotropic (external-mode) step of the INMSOM ocean model.

The product is the CUDA library libinmsom_gpu.so (C ABI in
include/inmsom_gpu.h); this package holds its sources (csrc/), its build
recipe, a ctypes binding, a host-side mirror of the reference interface and
seeded synthetic basins.
"""
from .grid import Basin, Bounds, Consts
from ._lib import InmsomError

__all__ = ["Basin", "Bounds", "Consts", "InmsomError"]
