"""ctypes wrapper of the CPU oracle (oracle/_build/libhsoracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU legs of bench.py, never by the product package.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _build.LIB
        if not os.path.exists(path):
            path = _build.build()
        l = C.CDLL(path)
        P = C.POINTER
        I, D = C.c_int, C.c_double
        pI, pD, pU8, pL = P(C.c_int), P(C.c_double), P(C.c_ubyte), P(C.c_long)
        sig = {
            "oracle_time_grid": (C.c_long, [D, D, pD, C.c_long]),
            "oracle_expm": (I, [I, pD, pD]),
            "oracle_krylov_expm": (I, [I, pI, pI, pD, D, pD, D, I, pD]),
            "oracle_st_unitary": (C.c_long, [I, pI, I, I, pI, pI, pD]),
            "oracle_trace_samples": (I, [D, pD, I, I, I, pD]),
            "oracle_st_flip_bits": (I, [D, I, C.c_ulonglong, D, pD, I, I, pU8]),
            "oracle_st_flip_bits_multi": (I, [D, I, C.c_ulonglong, pD, I, pD, I, I, pU8]),
            "oracle_apply_st": (I, [I, pI, pI, pD, D, D, C.c_uint, I, pD]),
            "oracle_hs_stochastic": (I, [I, I, pI, pI, pD, pI, pI, pD, D, pD, pD, I, I, I, pI, pI, pD, D, I, D, I,
                                         C.c_ulonglong, pU8, I, pI, pL, pI, pD, pD, pD, pD, pD, I]),
            "oracle_yield_correction": (D, [D, D]),
        }
        for name, (res, args) in sig.items():
            f = getattr(l, name)
            f.restype = res
            f.argtypes = args
        _lib = l
    return _lib


def _p(a, t):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(t))


def _cplx(a):
    return np.ascontiguousarray(a, dtype=np.complex128).view(np.float64)


def time_grid(total: float, dt: float) -> np.ndarray:
    n = lib().oracle_time_grid(total, dt, None, 0)
    t = np.zeros(n)
    lib().oracle_time_grid(total, dt, _p(t, C.c_double), n)
    return t


def expm(A: np.ndarray) -> np.ndarray:
    n = A.shape[0]
    a = np.ascontiguousarray(np.asarray(A, dtype=np.complex128).T).view(np.float64)
    out = np.zeros((n, n), dtype=np.complex128)
    rc = lib().oracle_expm(n, _p(a, C.c_double), _p(out.view(np.float64), C.c_double))
    assert rc == 0
    return out.T


def krylov_expm(H_csr, kappa: float, b: np.ndarray, dt: float, m: int) -> np.ndarray:
    rowptr, col, val = H_csr
    D = len(rowptr) - 1
    out = np.zeros(D, dtype=np.complex128)
    lib().oracle_krylov_expm(D, _p(np.ascontiguousarray(rowptr, np.int32), C.c_int),
                             _p(np.ascontiguousarray(col, np.int32), C.c_int), _p(_cplx(val), C.c_double),
                             kappa, _p(_cplx(b), C.c_double), dt, m, _p(out.view(np.float64), C.c_double))
    return out


def st_unitary(dims: list[int], e1: int, e2: int):
    d = np.asarray(dims, dtype=np.int32)
    nnz = lib().oracle_st_unitary(len(dims), _p(d, C.c_int), e1, e2, None, None, None)
    D = int(np.prod(dims))
    rowptr = np.zeros(D + 1, np.int32)
    col = np.zeros(nnz, np.int32)
    val = np.zeros(nnz, np.complex128)
    lib().oracle_st_unitary(len(dims), _p(d, C.c_int), e1, e2, _p(rowptr, C.c_int), _p(col, C.c_int),
                            _p(val.view(np.float64), C.c_double))
    return rowptr, col, val


def trace_samples(seed: float, fixed: np.ndarray, Z: int, M: int) -> np.ndarray:
    F = len(fixed)
    out = np.zeros((M, F * Z), dtype=np.complex128)
    lib().oracle_trace_samples(seed, _p(_cplx(fixed), C.c_double), F, Z, M, _p(out.view(np.float64), C.c_double))
    return out.T


def st_flip_bits(seed: float, seed_mode: int, orientation: int, event_rate: float, times, M: int) -> np.ndarray:
    t = np.ascontiguousarray(times, np.float64)
    bits = np.zeros(max(1, ((len(t) - 1) * 2 * M + 7) // 8), np.uint8)
    lib().oracle_st_flip_bits(seed, seed_mode, orientation, event_rate, _p(t, C.c_double), len(t), M,
                              _p(bits, C.c_ubyte))
    return bits


def st_flip_bits_multi(seed: float, seed_mode: int, orientation: int, event_rates, times, M: int) -> np.ndarray:
    """Flip bits of several dephasing terms on one electron pair (superposed-Poisson branch)."""
    t = np.ascontiguousarray(times, np.float64)
    r = np.ascontiguousarray(event_rates, np.float64)
    bits = np.zeros(max(1, ((len(t) - 1) * 2 * M + 7) // 8), np.uint8)
    rc = lib().oracle_st_flip_bits_multi(seed, seed_mode, orientation, _p(r, C.c_double), len(r), _p(t, C.c_double),
                                         len(t), M, _p(bits, C.c_ubyte))
    if rc:
        raise ValueError("oracle flip stream failed")
    return bits


def apply_st(U_csr, event_rate: float, dt: float, seed: int, factors: np.ndarray) -> np.ndarray:
    """One ApplyStochasticRelaxationHilbert call with std::mt19937(seed); factors D x M."""
    rowptr, col, val = U_csr
    D, M = factors.shape
    buf = np.array(np.asarray(factors, np.complex128).T, order="C", copy=True)
    rc = lib().oracle_apply_st(D, _p(np.ascontiguousarray(rowptr, np.int32), C.c_int),
                               _p(np.ascontiguousarray(col, np.int32), C.c_int), _p(_cplx(val), C.c_double),
                               event_rate, dt, seed, M, _p(buf.view(np.float64), C.c_double))
    assert rc == 0
    return buf.T


def hs_stochastic(H_csr, factors: np.ndarray, times, observables, *, kappa: float = 0.0, K_csr=None,
                  method: int = 0, krylov: int = 16, U_csr=None, event_rate: float = 0.0, noise_mode: int = 0,
                  seed: float = 1.0, seed_mode: int = 0, orientation: int = 0, flip_bits=None, nthreads: int = 1):
    """Full stochastic loop for one orientation.

    observables: list of (CSR, rate).  Returns dict with values [(ntimes) x nobs],
    traj_yield [M x nobs], yield [nobs], factors (final, D x M)."""
    rowptr, col, val = H_csr
    D = len(rowptr) - 1
    F = np.asarray(factors, np.complex128)
    M = F.shape[1]
    buf = np.array(F.T, dtype=np.complex128, order="C", copy=True)  # the oracle works in place
    t = np.ascontiguousarray(times, np.float64)
    nobs = len(observables)
    orow = np.concatenate([np.asarray(o[0][0], np.int32) for o in observables])
    off = np.zeros(nobs, dtype=np.int64)
    acc = 0
    for i, o in enumerate(observables):
        off[i] = acc
        acc += len(o[0][1])
    ocol = np.ascontiguousarray(np.concatenate([np.asarray(o[0][1], np.int32) for o in observables]))
    oval = _cplx(np.concatenate([np.asarray(o[0][2], np.complex128) for o in observables]))
    rates = np.ascontiguousarray([float(o[1]) for o in observables], np.float64)
    values = np.zeros((len(t), nobs))
    traj = np.zeros((M, nobs))
    yld = np.zeros(nobs)
    if K_csr is not None:
        kr, kc, kv = (np.ascontiguousarray(K_csr[0], np.int32), np.ascontiguousarray(K_csr[1], np.int32),
                      _cplx(K_csr[2]))
    else:
        kr = kc = kv = None
    if U_csr is not None:
        ur, uc, uv = (np.ascontiguousarray(U_csr[0], np.int32), np.ascontiguousarray(U_csr[1], np.int32),
                      _cplx(U_csr[2]))
    else:
        ur = uc = uv = None
    fb = None if flip_bits is None else np.ascontiguousarray(flip_bits, np.uint8)
    rc = lib().oracle_hs_stochastic(
        D, M, _p(np.ascontiguousarray(rowptr, np.int32), C.c_int), _p(np.ascontiguousarray(col, np.int32), C.c_int),
        _p(_cplx(val), C.c_double), _p(kr, C.c_int), _p(kc, C.c_int), _p(kv, C.c_double), kappa,
        _p(buf.view(np.float64), C.c_double), _p(t, C.c_double), len(t), method, krylov, _p(ur, C.c_int),
        _p(uc, C.c_int), _p(uv, C.c_double), event_rate, noise_mode, seed, seed_mode, orientation,
        _p(fb, C.c_ubyte), nobs, _p(np.ascontiguousarray(orow), C.c_int), _p(off.astype(np.int64), C.c_long),
        _p(ocol, C.c_int), _p(oval, C.c_double), _p(rates, C.c_double), _p(values, C.c_double),
        _p(traj, C.c_double), _p(yld, C.c_double), nthreads)
    if rc != 0:
        raise RuntimeError(f"oracle_hs_stochastic failed ({rc})")
    return {"values": values, "traj_yield": traj, "yield": yld, "factors": buf.T}


def yield_correction(total: float, kmax: float) -> float:
    return lib().oracle_yield_correction(total, kmax)
