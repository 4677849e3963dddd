"""B200-native MLS-MPM fluid substep and diffuse spray/foam update.

Drop-in for the compute side of the reference's fluid-gpu.js / diffuse-gpu.js:
the C ABI in include/mpm_b200.h (libmpm_b200.so, CUDA sm_100a) and, over it,
FluidGPU / DiffuseGPU classes with the reference's method names.
"""
from . import abi, host, scenes
from .abi import MpmError, load_library
from .fluid_gpu import DiffuseGPU, FluidGPU

__all__ = ["abi", "host", "scenes", "load_library", "MpmError", "FluidGPU", "DiffuseGPU"]
