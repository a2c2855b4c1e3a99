"""Host-side mirror of MolSpin's HSGeneral stochastic interface for the B200 path.

The reference runs, per orientation, the loop of
``TaskHSGeneral::RunLocal`` (RunSection/General/HS/TaskHSGeneral.cpp:471-560):
``HSObservableCollector::Evaluate`` then ``HSPropagator::StepStochastic`` at
every point of the exact-endpoint time grid, followed by
``HSObservableCollector::IntegrateFiniteTime`` and the optional
``ApplyFiniteTimeYieldCorrection``.  Here that loop is one call into the
msgpu C ABI (include/msgpu.h); this module keeps the reference's vocabulary:

* :class:`HSExecutionPlan` -- the task keys that select and shape the path
  (HSExecutionPlan.h:33-117 defaults), plus the backend keys
  ``accelerator``/``gpuprecision``/``noise``;
* :class:`HSPropagatorB200` -- the propagator backend: owns a device context,
  takes H / K / the singlet-triplet cache / the observables, and propagates a
  factor block (replaces ``HSPropagator::StepStochastic`` and the per-step
  ``Evaluate``);
* :func:`run_stochastic_yields` -- ``RunLocal`` for one orientation and one
  spin system: trace sampling, propagation, integration, yield correction.

Errors are raised as :class:`MsgpuError` carrying the library's message,
the analogue of the reference's ``bool`` + ``std::string &error`` returns.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .systems import SpinSystem, time_grid


class MsgpuError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"msgpu error {code}: {message}")
        self.code = code


@dataclass
class HSExecutionPlan:
    """Subset of RunSection/General/HS/HSExecutionPlan.h for sampling=stochastic."""
    totaltime: float = 10000.0
    timestep: float = 1.0
    krylovsize: int = 16
    montecarlosamples: int = 1
    seed: float = 1.0
    yieldcorrections: bool = False
    # backend selection (new optional task keys)
    accelerator: str = "b200"
    gpuprecision: str = "c128"        # "c128" (plain) | "c64" (precision form)
    noise: str = "reference"          # "reference" (mt19937 replay) | "philox"

    def validate(self):
        if not (math.isfinite(self.totaltime) and self.totaltime >= 0.0):
            raise ValueError("totaltime must be finite and non-negative")
        if not (math.isfinite(self.timestep) and self.timestep > 0.0):
            raise ValueError("timestep must be finite and positive")
        if self.krylovsize < 1:
            self.krylovsize = 16  # HSExecutionPlan.cpp:413-414
        if self.montecarlosamples < 1:
            raise ValueError("montecarlosamples must be at least one")
        if self.gpuprecision not in ("c128", "c64"):
            raise ValueError("gpuprecision must be c128 or c64")
        if self.noise not in ("reference", "philox"):
            raise ValueError("noise must be reference or philox")


def _check(ctx, rc: int):
    if rc != L.MSGPU_OK:
        msg = L.lib.msgpu_last_error(ctx)
        raise MsgpuError(rc, msg.decode() if msg else "unknown")


class HSPropagatorB200:
    """Device context holding one spin system's H, K, noise and observables."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        self.ctx = L.lib.msgpu_create(int(device), int(hbm_budget))
        if not self.ctx:
            raise MsgpuError(L.MSGPU_ERR_CUDA, f"cannot create a context on CUDA device {device}")
        self.D = 0
        self.M = 0
        self.nobs = 0

    def close(self):
        if self.ctx:
            L.lib.msgpu_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------ inputs
    def set_hamiltonian(self, rowptr, col, val):
        rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        col = np.ascontiguousarray(col, dtype=np.int32)
        v = L.as_interleaved(val)
        D = len(rowptr) - 1
        _check(self.ctx, L.lib.msgpu_upload_hamiltonian_csr(self.ctx, D, L.iptr(rowptr), L.iptr(col), L.dptr(v)))
        self.D = D

    def set_hamiltonian_terms(self, rowptr, col, vals, coef):
        """H = sum_k coef_k H_k on one CSR pattern (vals: nterms x nnz complex);
        later field changes go through set_hamiltonian_coefficients."""
        rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        col = np.ascontiguousarray(col, dtype=np.int32)
        v = np.ascontiguousarray(np.asarray(vals, dtype=np.complex128))
        c = np.ascontiguousarray(coef, dtype=np.float64)
        D = len(rowptr) - 1
        _check(self.ctx, L.lib.msgpu_upload_hamiltonian_terms(self.ctx, D, L.iptr(rowptr), L.iptr(col), v.shape[0],
                                                              L.dptr(v.view(np.float64).reshape(-1)), L.dptr(c)))
        self.D = D

    def set_hamiltonian_coefficients(self, coef):
        c = np.ascontiguousarray(coef, dtype=np.float64)
        _check(self.ctx, L.lib.msgpu_set_hamiltonian_coefficients(self.ctx, L.dptr(c)))

    def set_hamiltonian_schedule(self, coef, first_step: int = 0):
        """coef: (nsteps, nterms) coefficients, row j for global step first_step + j
        (H at that step's midpoint); None clears the schedule."""
        if coef is None:
            _check(self.ctx, L.lib.msgpu_set_hamiltonian_schedule(self.ctx, None, 0, 0))
            return
        c = np.ascontiguousarray(coef, dtype=np.float64)
        _check(self.ctx, L.lib.msgpu_set_hamiltonian_schedule(self.ctx, L.dptr(c.reshape(-1)), int(first_step),
                                                              int(c.shape[0])))

    def set_hamiltonian_schedule_rk4(self, coef, first_step: int = 0):
        """coef: (2 nsteps + 1, nterms) coefficients for the RK4 propagator with a
        time-dependent H: row 2j at the start of global step first_step + j, row
        2j + 1 at its midpoint, row 2j + 2 at its end; None clears the schedule."""
        if coef is None:
            _check(self.ctx, L.lib.msgpu_set_hamiltonian_schedule_rk4(self.ctx, None, 0, 0))
            return
        c = np.ascontiguousarray(coef, dtype=np.float64)
        if c.shape[0] < 3 or c.shape[0] % 2 != 1:
            raise ValueError("an RK4 schedule has 2 nsteps + 1 rows")
        _check(self.ctx, L.lib.msgpu_set_hamiltonian_schedule_rk4(self.ctx, L.dptr(c.reshape(-1)), int(first_step),
                                                                  int((c.shape[0] - 1) // 2)))

    def set_reaction(self, kappa: float | None = None, csr=None):
        if csr is None:
            _check(self.ctx, L.lib.msgpu_set_reaction_scalar(self.ctx, float(kappa)))
        else:
            rowptr, col, val = csr
            rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
            col = np.ascontiguousarray(col, dtype=np.int32)
            _check(self.ctx, L.lib.msgpu_upload_reaction_csr(self.ctx, L.iptr(rowptr), L.iptr(col),
                                                             L.dptr(L.as_interleaved(val))))

    def set_electron_pair(self, stride1: int, stride2: int):
        _check(self.ctx, L.lib.msgpu_set_electron_pair(self.ctx, int(stride1), int(stride2)))

    def set_observables(self, obs: list[tuple[np.ndarray, float]]):
        _check(self.ctx, L.lib.msgpu_clear_observables(self.ctx))
        for op, rate in obs:
            a = L.as_interleaved(np.asarray(op, dtype=np.complex128).reshape(4, 4))
            _check(self.ctx, L.lib.msgpu_add_pair_observable(self.ctx, L.dptr(a), float(rate)))
        self.nobs = len(obs)

    def set_noise(self, st_rate: float, mode: int, seed: int = 0, bits: np.ndarray | None = None,
                  nsteps: int = 0, ntraj: int = 0):
        b = None if bits is None else np.ascontiguousarray(bits, dtype=np.uint8)
        _check(self.ctx, L.lib.msgpu_set_st_noise(self.ctx, float(st_rate), int(mode), int(seed) & ((1 << 64) - 1),
                                                  L.u8ptr(b), int(nsteps), int(ntraj)))

    def set_factors(self, factors: np.ndarray):
        """factors: D x M complex (any layout); column j is trajectory j."""
        F = np.asarray(factors, dtype=np.complex128)
        D, M = F.shape
        buf = np.ascontiguousarray(F.T)  # M x D C-order == D x M column-major
        _check(self.ctx, L.lib.msgpu_upload_factors(self.ctx, D, M, L.dptr(buf.view(np.float64))))
        self.M = M

    def get_factors(self) -> np.ndarray:
        out = np.zeros((self.M, self.D), dtype=np.complex128)
        _check(self.ctx, L.lib.msgpu_download_factors(self.ctx, L.dptr(out.view(np.float64))))
        return out.T

    # ------------------------------------------------------------ propagation
    PRECISIONS = {"c128": L.PREC_C128, "c64": L.PREC_C64, "bf16x3": L.PREC_BF16X3, "bf16x6": L.PREC_BF16X6,
                  "int8x4": L.PREC_INT8X4}

    def propagate(self, times: np.ndarray, krylov: int, precision: str = "c128", step_offset: int = 0,
                  accumulate: bool = False, recurrence: int = L.REC_AUTO, propagator: str = "krylov"):
        """propagator "krylov" (precision c128 | c64), "dense" (bf16x3 | bf16x6 | int8x4,
        tensor cores), "taylor" (c128; the reference's autoexpm) or "rk4" (c128, explicit)."""
        t = np.ascontiguousarray(times, dtype=np.float64)
        prop = {"krylov": L.PROP_KRYLOV, "dense": L.PROP_DENSE, "taylor": L.PROP_TAYLOR, "rk4": L.PROP_RK4}[propagator]
        p = L.RunParams(L.dptr(t), len(t), int(krylov), self.PRECISIONS[precision], int(recurrence), prop,
                        int(step_offset), 1 if accumulate else 0)
        _check(self.ctx, L.lib.msgpu_run(self.ctx, C.byref(p)))
        self._last_ntimes = len(t)

    def yields(self):
        per = np.zeros((self.M, self.nobs), dtype=np.float64)
        ens = np.zeros(self.nobs, dtype=np.float64)
        _check(self.ctx, L.lib.msgpu_fetch_yields(self.ctx, L.dptr(per), L.dptr(ens)))
        return per, ens

    def values(self):
        v = np.zeros((self._last_ntimes, self.nobs), dtype=np.float64)
        _check(self.ctx, L.lib.msgpu_fetch_values(self.ctx, L.dptr(v)))
        return v

    def set_option(self, key: int, value: float):
        _check(self.ctx, L.lib.msgpu_set_option(self.ctx, int(key), float(value)))

    def get_option(self, key: int) -> float:
        v = C.c_double(0.0)
        _check(self.ctx, L.lib.msgpu_get_option(self.ctx, int(key), C.byref(v)))
        return v.value

    def spmm_choice(self) -> dict:
        """The quartet SpMM the last complex64 streamed run used: variant, quartet
        tile and trajectory groups (msgpu_spmm_choice; variant -1 before any run)."""
        v, t, g = C.c_int(0), C.c_int(0), C.c_int(0)
        _check(self.ctx, L.lib.msgpu_spmm_choice(self.ctx, C.byref(v), C.byref(t), C.byref(g)))
        return {"spmm_variant": v.value, "spmm_tile": t.value, "traj_groups": g.value}

    def set_form(self, form: str | int):
        """"auto" | "streamed" | "resident" (see MSGPU_FORM_* in include/msgpu.h)."""
        codes = {"auto": L.FORM_AUTO, "streamed": L.FORM_STREAMED, "resident": L.FORM_RESIDENT}
        _check(self.ctx, L.lib.msgpu_set_form(self.ctx, codes[form] if isinstance(form, str) else int(form)))

    def launch_count(self) -> int:
        return int(L.lib.msgpu_launch_count(self.ctx))

    def profile(self, enable: bool | int = True):
        """True/1: time every launch; 2: sampled (every 32nd time step, every 8th dense GEMM); False/0: off."""
        mode = int(enable) if not isinstance(enable, bool) else (1 if enable else 0)
        _check(self.ctx, L.lib.msgpu_profile_enable(self.ctx, mode))

    def profile_read(self, cls: int):
        ms = C.c_double(0.0)
        n = C.c_longlong(0)
        _check(self.ctx, L.lib.msgpu_profile_read(self.ctx, int(cls), C.byref(ms), C.byref(n)))
        return ms.value, n.value


def reference_flip_bits_multi(seed: float, st_rates, times: np.ndarray, M: int, orientation: int = 0,
                              seed_mode: int = 0) -> np.ndarray:
    """The reference's flip stream for several dephasing Operators on the same
    electron pair (st_rates: each Operator's rate), as parity bits; replay with
    st_rate = sum(st_rates)."""
    t = np.ascontiguousarray(times, dtype=np.float64)
    r = np.ascontiguousarray(st_rates, dtype=np.float64)
    bits = np.zeros(max(1, ((len(t) - 1) * 2 * M + 7) // 8), dtype=np.uint8)
    rc = L.lib.msgpu_host_reference_flip_bits_multi(float(seed), int(seed_mode), int(orientation), L.dptr(r), len(r),
                                                    L.dptr(t), len(t), int(M), L.u8ptr(bits))
    if rc:
        raise ValueError("flip stream generation failed")
    return bits


def reference_flip_bits(seed: float, st_rate: float, times: np.ndarray, M: int, orientation: int = 0,
                        seed_mode: int = 0) -> np.ndarray:
    """The reference's singlet-triplet flip stream for one orientation, as bits."""
    t = np.ascontiguousarray(times, dtype=np.float64)
    nb = ((len(t) - 1) * 2 * M + 7) // 8
    bits = np.zeros(max(1, nb), dtype=np.uint8)
    rc = L.lib.msgpu_host_reference_flip_bits(float(seed), int(seed_mode), int(orientation), float(st_rate),
                                              L.dptr(t), len(t), int(M), L.u8ptr(bits))
    if rc:
        raise ValueError("flip stream generation failed")
    return bits


def philox_flip_bits(seed: int, st_rate: float, times: np.ndarray, M: int, traj_offset: int = 0,
                     step_offset: int = 0) -> np.ndarray:
    t = np.ascontiguousarray(times, dtype=np.float64)
    nb = ((len(t) - 1) * 2 * M + 7) // 8
    bits = np.zeros(max(1, nb), dtype=np.uint8)
    L.lib.msgpu_host_philox_flip_bits(int(seed), int(traj_offset), int(step_offset), float(st_rate), L.dptr(t),
                                      len(t), int(M), L.u8ptr(bits))
    return bits


def yield_correction(totaltime: float, kmax: float) -> float:
    """1/(1 - exp(-T kmax)) (HSObservableCollector.cpp:361-392)."""
    d = 1.0 - math.exp(-totaltime * kmax)
    if not (d > 0.0 and math.isfinite(d)):
        raise ValueError("yieldcorrections=true requires a positive finite total time and rate")
    return 1.0 / d


def run_stochastic_yields(system: SpinSystem, plan: HSExecutionPlan, device: int = 0, orientation: int = 0,
                          factors: np.ndarray | None = None, hbm_budget: int = 0) -> dict:
    """TaskHSGeneral::RunLocal for one spin system at one orientation, calculation=yields.

    Returns the ensemble yields (one per sink, rate-weighted as transition
    yields), the per-trajectory yields of the columns actually propagated
    (trajectory j of factors / sqrt(M)) and the per-time-point values."""
    plan.validate()
    times = time_grid(plan.totaltime, plan.timestep)
    M = plan.montecarlosamples
    if factors is None:
        factors = system.trace_samples(M, plan.seed)
    rowptr, col, val = system.hamiltonian_csr()
    obs = system.observables()
    with HSPropagatorB200(device, hbm_budget) as prop:
        prop.set_hamiltonian(rowptr, col, val)
        prop.set_reaction(kappa=system.kappa())
        prop.set_electron_pair(*system.electron_strides())
        prop.set_observables([(op, rate) for _, op, rate in obs])
        if system.st_rate > 0.0:
            if plan.noise == "reference":
                bits = reference_flip_bits(plan.seed, system.st_rate, times, M, orientation)
                prop.set_noise(system.st_rate, L.NOISE_REPLAY, 0, bits, len(times) - 1, M)
            else:
                prop.set_noise(system.st_rate, L.NOISE_PHILOX, int(plan.seed) * 1_000_003 + orientation)
        prop.set_factors(factors)
        prop.propagate(times, plan.krylovsize, plan.gpuprecision)
        per, ens = prop.yields()
        values = prop.values()
    if plan.yieldcorrections:
        kmax = max(rate for _, _, rate in obs)
        c = yield_correction(plan.totaltime, kmax)
        ens = ens * c
        per = per * c
    return {"names": [n for n, _, _ in obs], "yields": ens, "traj_yields": per, "values": values, "times": times}


def run_powder_yields(system: SpinSystem, plan: HSExecutionPlan, field_T: float, directions: np.ndarray,
                      weights: np.ndarray | None = None, device: int = 0, factors: np.ndarray | None = None,
                      hbm_budget: int = 0) -> dict:
    """The orientation loop of TaskHSGeneral::RunLocal (TaskHSGeneral.cpp:347-575)
    for a field of strength field_T (T) along each unit vector of `directions`.

    One device context holds H as fixed-pattern terms (H_0 + Bx Zx + By Zy +
    Bz Zz, systems.field_terms); each orientation only changes the field
    coefficients on the device.  Every orientation starts from the same
    trace samples (a copy of the prepared factors, TaskHSGeneral.cpp:359) and
    draws its own noise stream; the ensemble yields are averaged with the
    weights (uniform when omitted), TaskHSGeneral.cpp:568-575.  The system's
    own Zeeman terms are replaced by the orientation's field."""
    plan.validate()
    dirs = np.asarray(directions, dtype=np.float64).reshape(-1, 3)
    w = np.full(len(dirs), 1.0 / len(dirs)) if weights is None else np.asarray(weights, dtype=np.float64)
    times = time_grid(plan.totaltime, plan.timestep)
    M = plan.montecarlosamples
    if factors is None:
        factors = system.trace_samples(M, plan.seed)
    from .systems import field_terms
    rowptr, col, vals = field_terms(system)
    obs = system.observables()
    per_orientation = []
    with HSPropagatorB200(device, hbm_budget) as prop:
        prop.set_hamiltonian_terms(rowptr, col, vals, [1.0, *(field_T * dirs[0])])
        prop.set_reaction(kappa=system.kappa())
        prop.set_electron_pair(*system.electron_strides())
        prop.set_observables([(op, rate) for _, op, rate in obs])
        for i, d in enumerate(dirs):
            prop.set_hamiltonian_coefficients([1.0, *(field_T * d)])
            if system.st_rate > 0.0:
                if plan.noise == "reference":
                    bits = reference_flip_bits(plan.seed, system.st_rate, times, M, i)
                    prop.set_noise(system.st_rate, L.NOISE_REPLAY, 0, bits, len(times) - 1, M)
                else:
                    prop.set_noise(system.st_rate, L.NOISE_PHILOX, int(plan.seed) * 1_000_003 + i)
            prop.set_factors(factors)
            prop.propagate(times, plan.krylovsize, plan.gpuprecision)
            per_orientation.append(prop.yields()[1])
    ens = np.asarray(per_orientation)
    if plan.yieldcorrections:
        ens = ens * yield_correction(plan.totaltime, max(rate for _, _, rate in obs))
    return {"names": [n for n, _, _ in obs], "yields": w @ ens, "orientation_yields": ens, "weights": w}
