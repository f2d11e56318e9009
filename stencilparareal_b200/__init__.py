"""B200-native (sm_100a) advection-diffusion propagator and Parareal driver.

A from-scratch implementation of the hot path of andyspiros/StencilParareal:
class Convection (src/Convection) and class Parareal (src/Parareal), behind a
C ABI (include/sp_abi.h) implemented by ``libstencilparareal.so``.
"""
from . import _lib
from ._lib import SP_COARSE_EULER, SP_COARSE_RK4, SP_F32, SP_F64, SpError
from .convection import Convection, ConvectionField, launch_count, layout
from .parareal import Parareal, RuntimeConfiguration

__all__ = ["Convection", "ConvectionField", "Parareal", "RuntimeConfiguration", "SpError", "SP_F64", "SP_F32",
           "SP_COARSE_EULER", "SP_COARSE_RK4", "launch_count", "layout", "_lib"]
