"""B200-native compressible staggered-grid fluctuating hydrodynamics step.

Drop-in for FHDeX's ``RK3stepStag`` path: sm_100a CUDA kernels behind the C ABI
in ``include/fhd_capi.h`` (``fhdex_b200/lib/libfhd_b200.so``), with this Python
package as a host-side mirror of the reference interface.
"""
from .params import Params, argon, argon_single, mixture4, parse_inputs, stable_dt  # noqa: F401
from .state import StagState, StepNoise  # noqa: F401

__all__ = ["Params", "argon", "argon_single", "mixture4", "parse_inputs", "stable_dt", "StagState", "StepNoise"]
