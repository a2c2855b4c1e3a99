"""ctypes binding of libmsgpu.so (include/msgpu.h, include/msgpu_host.h).

The library is the product: there is no fallback.  If libmsgpu.so is missing
or cannot be loaded, importing this module raises immediately.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmsgpu.so")

MSGPU_OK = 0
MSGPU_ERR_INVALID = 1
MSGPU_ERR_BUDGET = 2
MSGPU_ERR_NONFINITE = 3
MSGPU_ERR_EXPM = 4
MSGPU_ERR_CUDA = 6
MSGPU_ERR_STATE = 7
MSGPU_ERR_SCRATCH = 8
NOALLOC_SCRATCH_BYTES = 16 << 20

PREC_C128 = 0
PREC_C64 = 1
REC_AUTO = 0
REC_ARNOLDI = 1
REC_LANCZOS = 2
PROP_KRYLOV = 0
PROP_DENSE = 1
PROP_TAYLOR = 2
PROP_RK4 = 3
OPT_TAYLOR_TOL = 2
OPT_SPMM_VARIANT = 3
OPT_LANCZOS_CLUSTER = 4
OPT_TRAJ_GROUPS = 5
OPT_COMBINE_TILE = 6
PREC_BF16X3 = 2
PREC_BF16X6 = 3
PREC_INT8X4 = 4
OPT_DENSE_RENORMALIZE = 1
NOISE_NONE = 0
NOISE_REPLAY = 1
NOISE_PHILOX = 2
FORM_AUTO = 0
FORM_STREAMED = 1
FORM_RESIDENT = 2

KC_APPLY, KC_ORTH, KC_REDUCE, KC_EXPM, KC_COMBINE, KC_YIELD, KC_GEMM, KC_LANCZOS = range(8)


class RunParams(C.Structure):
    _fields_ = [
        ("times", C.POINTER(C.c_double)),
        ("ntimes", C.c_int),
        ("krylov_dim", C.c_int),
        ("precision", C.c_int),
        ("recurrence", C.c_int),
        ("propagator", C.c_int),
        ("step_offset", C.c_longlong),
        ("accumulate", C.c_int),
    ]


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m molspin_b200.build` "
            "(the CUDA library is required; there is no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    P = C.c_void_p
    I = C.c_int
    D = C.c_double
    pI = C.POINTER(C.c_int)
    pD = C.POINTER(C.c_double)
    pU8 = C.POINTER(C.c_ubyte)
    sig = {
        "msgpu_create": (P, [I, C.c_size_t]),
        "msgpu_destroy": (None, [P]),
        "msgpu_last_error": (C.c_char_p, [P]),
        "msgpu_device_bytes": (C.c_size_t, [P]),
        "msgpu_set_stream": (I, [P, P]),
        "msgpu_upload_hamiltonian_csr": (I, [P, I, pI, pI, pD]),
        "msgpu_upload_hamiltonian_terms": (I, [P, I, pI, pI, I, pD, pD]),
        "msgpu_set_hamiltonian_coefficients": (I, [P, pD]),
        "msgpu_set_hamiltonian_schedule": (I, [P, pD, C.c_longlong, C.c_longlong]),
        "msgpu_set_hamiltonian_schedule_rk4": (I, [P, pD, C.c_longlong, C.c_longlong]),
        "msgpu_set_reaction_scalar": (I, [P, D]),
        "msgpu_upload_reaction_csr": (I, [P, pI, pI, pD]),
        "msgpu_set_electron_pair": (I, [P, I, I]),
        "msgpu_clear_observables": (I, [P]),
        "msgpu_add_pair_observable": (I, [P, pD, D]),
        "msgpu_set_st_noise": (I, [P, D, I, C.c_ulonglong, pU8, C.c_longlong, I]),
        "msgpu_upload_factors": (I, [P, I, I, pD]),
        "msgpu_upload_factors_device": (I, [P, I, I, P]),
        "msgpu_download_factors": (I, [P, pD]),
        "msgpu_run": (I, [P, C.POINTER(RunParams)]),
        "msgpu_fetch_yields": (I, [P, pD, pD]),
        "msgpu_fetch_values": (I, [P, pD]),
        "msgpu_profile_enable": (I, [P, I]),
        "msgpu_profile_read": (I, [P, I, pD, C.POINTER(C.c_longlong)]),
        "msgpu_launch_count": (C.c_longlong, [P]),
        "msgpu_set_form": (I, [P, I]),
        "msgpu_set_option": (I, [P, I, D]),
        "msgpu_get_option": (I, [P, I, pD]),
        "msgpu_batch_create": (P, [I, C.c_size_t]),
        "msgpu_batch_destroy": (None, [P]),
        "msgpu_batch_clear": (I, [P]),
        "msgpu_batch_last_error": (C.c_char_p, [P]),
        "msgpu_batch_add_system": (I, [P, I, pI, pI, pD, D, I, I, I, pD, pD, D, C.c_ulonglong, I, pD]),
        "msgpu_batch_tune": (I, [P, pD, I, I]),
        "msgpu_batch_run": (I, [P, pD, I, I, C.c_longlong, I]),
        "msgpu_batch_fetch_yields": (I, [P, I, pD, pD]),
        "msgpu_batch_stats": (I, [P, pD, pI, pI]),
        "msgpu_batch_launch_count": (C.c_longlong, [P]),
        "msgpu_spmm_choice": (I, [P, pI, pI, pI]),
        "msgpu_batch_system_info": (I, [P, I, pI, pI, pI, pI]),
        "msgpu_krylov_step_noalloc": (I, [I, P, P, P, D, I, P, P, D, I, P]),
        "msgpu_host_build_hamiltonian": (C.c_longlong, [I, pI, I, pI, pD, I, pI, pI, pD, pI, pI, pD]),
        "msgpu_host_trace_samples": (I, [D, pD, I, I, I, pD]),
        "msgpu_host_reference_flip_bits": (I, [D, I, C.c_ulonglong, D, pD, I, I, pU8]),
        "msgpu_host_reference_flip_bits_multi": (I, [D, I, C.c_ulonglong, pD, I, pD, I, I, pU8]),
        "msgpu_host_philox_flip_bits": (I, [C.c_ulonglong, C.c_uint, C.c_longlong, D, pD, I, I, pU8]),
        "msgpu_host_time_grid": (C.c_long, [D, D, pD, C.c_long]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def ptr(a: np.ndarray, ctype):
    """Pointer to a C-contiguous numpy array (None passes NULL)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(ctype))


def dptr(a):
    return ptr(a, C.c_double)


def iptr(a):
    return ptr(a, C.c_int)


def u8ptr(a):
    return ptr(a, C.c_ubyte)


def as_interleaved(z: np.ndarray) -> np.ndarray:
    """complex128 array -> contiguous float64 view (re, im interleaved)."""
    z = np.ascontiguousarray(z, dtype=np.complex128)
    return z.view(np.float64)
