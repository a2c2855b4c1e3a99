"""Batching form: many spin systems in one persistent launch.

The reference propagates the systems of a powder average or parameter sweep
one after another: the orientation loop of ``TaskHSGeneral::RunLocal``
(RunSection/General/HS/TaskHSGeneral.cpp:347) and the RunSection step loop
(main.cpp:651-678) each re-run the whole HSGeneral time loop.  Here every
(system, trajectory) pair of a system below the streamed-route dimension
(2048) advances inside ONE persistent kernel launch (msgpu_batch_* in
include/msgpu.h), replayed from a CUDA graph, with the team threshold and
grid size chosen by an autotuner on the batch.  Systems at or above that
dimension run the streamed precision form (quartet SpMM over the whole
trajectory block) on their own contexts and streams, concurrently with the
persistent launch: a persistent team propagates one trajectory at a time
and re-reads H per trajectory, which loses to the lockstep SpMM there.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .hsgeneral import MsgpuError
from .systems import SpinSystem


class BatchB200:
    def __init__(self, device: int = 0, hbm_budget: int = 0):
        self.b = L.lib.msgpu_batch_create(int(device), int(hbm_budget))
        if not self.b:
            raise MsgpuError(L.MSGPU_ERR_CUDA, f"cannot create a batch on CUDA device {device}")
        self.systems: list[tuple[int, int]] = []  # (M, nobs)

    def close(self):
        if self.b:
            L.lib.msgpu_batch_destroy(self.b)
            self.b = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != L.MSGPU_OK:
            raise MsgpuError(rc, L.lib.msgpu_batch_last_error(self.b).decode())

    def add(self, system: SpinSystem, factors: np.ndarray, seed: int) -> int:
        r, c, v = system.hamiltonian_csr()
        r = np.ascontiguousarray(r, np.int32)
        c = np.ascontiguousarray(c, np.int32)
        obs = system.observables()
        ops = np.ascontiguousarray(np.stack([np.asarray(op, np.complex128).reshape(4, 4) for _, op, _ in obs]))
        rates = np.ascontiguousarray([rate for _, _, rate in obs], np.float64)
        F = np.asarray(factors, np.complex128)
        D, M = F.shape
        buf = np.ascontiguousarray(F.T)
        s1, s2 = system.electron_strides()
        idx = L.lib.msgpu_batch_add_system(
            self.b, D, L.iptr(r), L.iptr(c), L.dptr(L.as_interleaved(v)), float(system.kappa()), s1, s2, len(obs),
            L.dptr(ops.view(np.float64).reshape(-1)), L.dptr(rates), float(system.st_rate), int(seed), M,
            L.dptr(buf.view(np.float64).reshape(-1)))
        if idx < 0:
            raise MsgpuError(-idx, L.lib.msgpu_batch_last_error(self.b).decode())
        self.systems.append((M, len(obs)))
        return idx

    def clear(self):
        """Drops every system; the device buffers of the persistent route are
        kept for the next add() calls (msgpu_batch_clear)."""
        self._check(L.lib.msgpu_batch_clear(self.b))
        self.systems.clear()

    def tune(self, times: np.ndarray, krylov: int):
        t = np.ascontiguousarray(times, np.float64)
        self._check(L.lib.msgpu_batch_tune(self.b, L.dptr(t), len(t), int(krylov)))

    def run(self, times: np.ndarray, krylov: int, step_offset: int = 0, accumulate: bool = False):
        t = np.ascontiguousarray(times, np.float64)
        self._check(L.lib.msgpu_batch_run(self.b, L.dptr(t), len(t), int(krylov), int(step_offset),
                                          1 if accumulate else 0))

    def yields(self, index: int):
        M, nobs = self.systems[index]
        per = np.zeros((M, nobs))
        ens = np.zeros(nobs)
        self._check(L.lib.msgpu_batch_fetch_yields(self.b, int(index), L.dptr(per), L.dptr(ens)))
        return per, ens

    def launch_count(self) -> int:
        return int(L.lib.msgpu_batch_launch_count(self.b))

    def system_info(self, i: int) -> dict:
        """Route of system i (streamed or persistent) and, when streamed, the
        SpMM its context's tuner picked."""
        st, v, t, g = C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(0)
        self._check(L.lib.msgpu_batch_system_info(self.b, int(i), C.byref(st), C.byref(v), C.byref(t), C.byref(g)))
        return {"streamed": bool(st.value), "spmm_variant": v.value, "spmm_tile": t.value, "traj_groups": g.value}

    def stats(self):
        ms = C.c_double(0.0)
        th = C.c_int(0)
        cps = C.c_int(0)
        self._check(L.lib.msgpu_batch_stats(self.b, C.byref(ms), C.byref(th), C.byref(cps)))
        return {"last_run_ms": ms.value, "team_threshold": th.value, "ctas_per_sm": cps.value}
