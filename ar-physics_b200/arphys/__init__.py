"""Host-side Python mirror of the `FluidSim` interface over libarphys.so.

The compute path is the CUDA library behind include/arphys.h; this package
only builds scene records and calls the C ABI through ctypes.
"""
from .abi import (PARTICLE_DTYPE, SOLID_DTYPE, MATERIAL_DTYPE, INTERACTION_DTYPE, INVALID, INTEGRATORS,
                  ArpError, load_library)
from .scenes import Scene
from .sim import FluidSim

__all__ = ["PARTICLE_DTYPE", "SOLID_DTYPE", "MATERIAL_DTYPE", "INTERACTION_DTYPE", "INVALID", "INTEGRATORS",
           "ArpError", "load_library", "Scene", "FluidSim"]
