"""B200-native ICLS hot path: Python mirror of the reference driver interface.

The compute runs in ``libicls_gpu.so`` (CUDA, sm_100a) behind the C ABI of
include/icls_gpu.h; this package only binds it.
"""
from .config import (BCY_INOUT, BCY_OUTOUT, BCY_PERIODIC, BCY_WALLS, NS_CNTR2, NS_WENO5,
                     CURV_MLP, CURV_STENCIL, FIELD_ID, FIELDS, FP32, FP64, HOUC5,
                     SPEED_CURV, SPEED_UNFM, WENO5, IclsConfig, IclsScalars, Workload,
                     combined, field_shape, inflow_profile, init_drops, initial_velocity, make_config,
                     multi_drop, rising_bubble, seeded_drops, solenoidal_velocity, static_drop, workload_velocity)
from .binding import LIB_PATH, Backend, IclsError, Solver, gpu_backend

__all__ = [
    "BCY_INOUT", "BCY_OUTOUT", "BCY_PERIODIC", "BCY_WALLS", "NS_CNTR2", "NS_WENO5", "inflow_profile",
    "CURV_MLP", "CURV_STENCIL", "FIELD_ID", "FIELDS", "FP32", "FP64", "HOUC5",
    "SPEED_CURV", "SPEED_UNFM", "WENO5", "IclsConfig", "IclsScalars", "Workload",
    "combined", "field_shape", "init_drops", "initial_velocity", "make_config", "multi_drop",
    "rising_bubble", "seeded_drops", "solenoidal_velocity", "static_drop", "workload_velocity", "LIB_PATH", "Backend", "IclsError",
    "Solver", "gpu_backend",
]
