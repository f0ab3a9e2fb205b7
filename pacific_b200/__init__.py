"""B200-native Grains3D DEM time step (linked-cell binning, 27-cell pair
search, sphere narrow phase, HookeMemory contact law with hashed tangential
history, deterministic force reduction, second-order leapfrog)."""
from .grains import (FP32_SPLIT, FP64, ContactError, Grains, GrainsError, MotionError,
                     OutOfGridError, SimulationError, library)

__all__ = ["FP64", "FP32_SPLIT", "Grains", "GrainsError", "SimulationError", "ContactError",
           "MotionError", "OutOfGridError", "library"]
