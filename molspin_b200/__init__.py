"""molspin_b200 -- B200-native HSGeneral stochastic Hilbert-space propagation.

The compute path is libmsgpu.so (CUDA, sm_100a) behind the C ABI in
include/msgpu.h; this package is its Python host mirror.
"""
from . import _lib  # noqa: F401  (loads libmsgpu.so; raises if it is missing)
from .hsgeneral import (HSExecutionPlan, HSPropagatorB200, MsgpuError, philox_flip_bits, reference_flip_bits,
                        run_stochastic_yields, yield_correction)
from .systems import SpinSystem, Workload, radical_pair, time_grid

__all__ = [
    "HSExecutionPlan", "HSPropagatorB200", "MsgpuError", "SpinSystem", "Workload", "philox_flip_bits",
    "radical_pair", "reference_flip_bits", "run_stochastic_yields", "time_grid", "yield_correction",
]
