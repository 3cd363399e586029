"""B200-native (sm_100a) channel timestep of DIABLO behind a C ABI.

The compute path is libdiablo_gpu.so (hand-written CUDA, see csrc/); this
package holds the host-side mirror of the reference's interface: run
parameters (params), the y-grid (grid), initial fields (ics), Fortran host
layouts (layout) and the ctypes binding of the library (channel).
"""
from .params import DiabloParams, PREC_FP64, PREC_FP32SPLIT, kelvin_helmholtz, turbulent_channel

__all__ = ["DiabloParams", "PREC_FP64", "PREC_FP32SPLIT", "kelvin_helmholtz", "turbulent_channel"]
