"""molspin_b200 -- B200-native HSGeneral stochastic Hilbert-space propagation.

The compute path is libmsgpu.so (CUDA, sm_100a) behind the C ABI in
include/msgpu.h; this package is its Python host mirror.  The library is
loaded by the first import of ``_lib`` (every module that computes imports
it, and so does the first use of a name exported here), which raises
ImportError when libmsgpu.so is missing: there is no CPU fallback.  Importing
the package alone does not load it, so ``python -m molspin_b200.build`` works
on a fresh checkout.
"""
from importlib import import_module

_EXPORTS = {
    **{n: ".hsgeneral" for n in ("HSExecutionPlan", "HSPropagatorB200", "MsgpuError", "philox_flip_bits",
                                 "reference_flip_bits", "run_stochastic_yields", "yield_correction")},
    **{n: ".systems" for n in ("SpinSystem", "Workload", "radical_pair", "time_grid")},
}

__all__ = [
    "HSExecutionPlan", "HSPropagatorB200", "MsgpuError", "SpinSystem", "Workload", "philox_flip_bits",
    "radical_pair", "reference_flip_bits", "run_stochastic_yields", "time_grid", "yield_correction",
]


def __getattr__(name):
    if name in _EXPORTS:
        return getattr(import_module(_EXPORTS[name], __name__), name)
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
