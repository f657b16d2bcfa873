"""B200-native PEnGUIn hydro step: PPM sweeps, FARGO orbital advection and a
planet potential on one GPU, behind the C ABI of include/penguin_b200.h.

The compute path is libpenguin_b200.so (hand-written sm_100a CUDA kernels);
importing the host mirror loads it and fails loudly when it is missing.
"""
from . import _lib  # noqa: F401
from .host import (Batch, GPU_output_reduction, Index_Shift, PenguinError, Planet, Run,  # noqa: F401
                   build_ic, bundle_sweep2D, bundle_sweep3D, dump_fields, get_dt, init_planet,
                   kick_drift_kick, label, params, planet_forces, rotate_rings, run_device_bytes,
                   Server, sweep_axis, to_physical, torque_norm, dump_name, write_para_file,
                   write_time_rows)

__all__ = [
    "Run", "Planet", "PenguinError", "params", "build_ic", "label", "dump_fields", "to_physical",
    "get_dt", "Index_Shift", "bundle_sweep2D", "bundle_sweep3D", "GPU_output_reduction",
    "init_planet", "planet_forces", "kick_drift_kick", "torque_norm", "sweep_axis", "rotate_rings", "Batch", "Server",
    "run_device_bytes", "dump_name", "write_para_file", "write_time_rows",
]
