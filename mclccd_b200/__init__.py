"""mclccd_b200: continuous collision detection (mclccd's BVHTree hot path) on B200.

The compute path is libmclccd_b200.so (hand-written sm_100a CUDA behind a C
ABI, include/mclccd_b200.h); this package is its Python host-side mirror.
"""
from .ccd import (BVHTree, CCDError, Options, narrow_phase_bulk, vjp_toi, lib, LIB_PATH,  # noqa: F401
                  PREC_FP64, PREC_FP32_CERTIFIED, MEM_HOST, MEM_DEVICE)

__all__ = ["BVHTree", "CCDError", "Options", "narrow_phase_bulk", "vjp_toi", "lib", "LIB_PATH",
           "PREC_FP64", "PREC_FP32_CERTIFIED", "MEM_HOST", "MEM_DEVICE"]
