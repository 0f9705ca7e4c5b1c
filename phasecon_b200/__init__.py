"""phasecon_b200 -- B200-native MBIR hot path of phasecon (sm_100a).

The compute runs in libmbirgpu.so (CUDA kernels behind a C ABI declared in
include/mbirgpu.h); this package is its Python-side mirror of the reference
interface plus seeded synthetic workloads.
"""
from .mbir import (EXPORTS, LIB_PATH, Batch, MbirError, Options, Problem, Session, default_options, get_options,
                   lib, reconstruct, reconstruct_batch, set_options)

__all__ = ["EXPORTS", "LIB_PATH", "Batch", "MbirError", "Options", "Problem", "Session", "default_options",
           "get_options", "lib", "reconstruct", "reconstruct_batch", "set_options"]
