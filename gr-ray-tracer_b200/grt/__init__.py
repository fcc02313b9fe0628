"""B200-native GR-ray-tracer hot path: Python host side over the C ABI.

Modules:
  abi        ctypes structs mirroring include/grt.h
  lib        the shared library binding and the Context class
  config     reference-format TOML writer
  torus      Fishbone-Moncrief torus inputs in the reference's NumPy format
  workloads  the benchmark workloads
"""

from .abi import (GEN_BLACKBODY, GEN_CUSTOM, GEN_POWER_LAW, MODE_DISK, MODE_IMAGE, PREC_FP64, PREC_MIXED,
                  RK4, RK45, Params, PhotonArrays, ProductArrays)

__all__ = ["Params", "PhotonArrays", "ProductArrays", "MODE_IMAGE", "MODE_DISK", "RK4", "RK45",
           "PREC_FP64", "PREC_MIXED", "GEN_BLACKBODY", "GEN_POWER_LAW", "GEN_CUSTOM"]
