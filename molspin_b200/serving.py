"""Serving form: continuous batching of field/orientation/system solves.

A request is one HSGeneral stochastic yield solve -- one radical-pair system
at one field orientation, as one RunSection step of the reference
(RunSection::Run -> TaskHSGeneral::RunLocal, main.cpp:651-678).  The engine
admits requests as they arrive, first-fit against a device-memory budget and
a number of slots.  Each admitted request gets its own msgpu context (its
own CUDA stream; the budget it reserved is enforced by the context), and
worker threads drive the C ABI with the GIL released, so requests that
arrive while others run are admitted as soon as slots and memory free up
and their kernels overlap on the device.  Latency (arrival -> yields on the
host) is reported as p50/p99 beside throughput.

Results do not depend on the mix: noise is counter-based Philox keyed by the
request's seed and each trajectory/step, reductions are two-phase in a fixed
order, and the SpMM tile chosen by the autotuner only changes how partial
sums are grouped (so a request agrees with its solo run to rounding).
"""
from __future__ import annotations

import math
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from .hsgeneral import HSPropagatorB200
from .systems import Workload


@dataclass
class Request:
    rid: int
    arrival: float          # seconds after the start of the stream
    workload: Workload
    seed: int = 0


@dataclass
class Result:
    rid: int
    dim: int
    traj_steps: int
    arrival: float
    admitted: float = 0.0
    finished: float = 0.0
    yields: np.ndarray = field(default_factory=lambda: np.zeros(0))
    reserved: int = 0
    error: str = ""

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def footprint(w: Workload, precision: str = "c64") -> int:
    """Upper bound of the device bytes one request's context allocates."""
    D, M, m = w.system.dim, w.M, min(w.krylov, w.system.dim)
    ldm = (M + 63) // 64 * 64
    n = D * ldm
    nnz = D * (3 + 2 * (len(w.system.mult) - 2))
    H = nnz * (4 + 16 + 8 + 8) + 4 * (D + 1)
    state = n * 16 + D * M * 16                  # complex128 state + staging
    if D <= 1024:                                  # resident form
        work = D * M * 16 + (w.steps + 1) * M * 8 * 4 + ldm * 64
    elif precision == "c64":
        # Lanczos basis + U, quartet-block H, partial sums, staging
        work = n * 8 * (m + 2) + D // 4 * (16 * (len(w.system.mult) + 1) * 16) + 3 * n + n * 16
    else:
        work = n * 16 * (m + 3) + 3 * n * 2
    per_traj = ldm * (8 * (3 * 4 + 8 + 2 * m) + 16 * m * m)
    return int(1.15 * (H + state + work + per_traj)) + (64 << 20)


class ServingEngine:
    def __init__(self, device: int = 0, hbm_budget: int = 64 << 30, slots: int = 8, precision: str = "c64"):
        self.device = device
        self.budget = hbm_budget
        self.slots = slots
        self.precision = precision
        self._lock = threading.Condition()
        self._reserved = 0
        self._running = 0
        self.max_concurrency = 0
        self.peak_reserved = 0

    def solve(self, req: Request, budget: int = 0) -> np.ndarray:
        """One request on its own context; returns the ensemble yields."""
        w = req.workload
        s = w.system
        F = s.trace_samples(w.M, w.seed)
        with HSPropagatorB200(self.device, budget) as p:
            p.set_hamiltonian(*s.hamiltonian_csr())
            p.set_reaction(kappa=s.kappa())
            p.set_electron_pair(*s.electron_strides())
            p.set_observables([(op, rate) for _, op, rate in s.observables()])
            if s.st_rate > 0.0:
                p.set_noise(s.st_rate, L.NOISE_PHILOX, req.seed)
            p.set_factors(F)
            p.propagate(w.times(), w.krylov, self.precision)
            _, ens = p.yields()
        return ens

    def _worker(self, req: Request, res: Result, t0: float):
        try:
            res.yields = self.solve(req, res.reserved)
        except Exception as e:  # noqa: BLE001 -- reported per request
            res.error = str(e)
        res.finished = time.perf_counter() - t0
        with self._lock:
            self._reserved -= res.reserved
            self._running -= 1
            self._lock.notify_all()

    def serve(self, requests: list[Request], realtime: bool = True) -> list[Result]:
        """Run a request stream; arrivals are honoured in wall-clock time when
        realtime, otherwise every request is available at t=0."""
        order = sorted(requests, key=lambda r: r.arrival)
        results = {r.rid: Result(r.rid, r.workload.system.dim, r.workload.M * r.workload.steps,
                                 r.arrival if realtime else 0.0, reserved=footprint(r.workload, self.precision))
                   for r in order}
        for r in order:
            if results[r.rid].reserved > self.budget:
                results[r.rid].error = "request larger than the device-memory budget"
        waiting: list[Request] = []
        threads = []
        t0 = time.perf_counter()
        i = 0
        with self._lock:
            while True:
                now = time.perf_counter() - t0
                while i < len(order) and (not realtime or order[i].arrival <= now):
                    if not results[order[i].rid].error:
                        waiting.append(order[i])
                    i += 1
                # first fit: admit every waiting request that fits the free slots and memory
                k = 0
                while k < len(waiting) and self._running < self.slots:
                    req = waiting[k]
                    res = results[req.rid]
                    if self._reserved + res.reserved <= self.budget:
                        waiting.pop(k)
                        self._reserved += res.reserved
                        self._running += 1
                        self.max_concurrency = max(self.max_concurrency, self._running)
                        self.peak_reserved = max(self.peak_reserved, self._reserved)
                        res.admitted = now
                        th = threading.Thread(target=self._worker, args=(req, res, t0), daemon=True)
                        th.start()
                        threads.append(th)
                    else:
                        k += 1
                if i >= len(order) and not waiting and self._running == 0:
                    break
                timeout = None
                if realtime and i < len(order):
                    timeout = max(0.0, order[i].arrival - (time.perf_counter() - t0))
                self._lock.wait(timeout=timeout if timeout is not None else 1.0)
        for th in threads:
            th.join()
        return [results[r.rid] for r in requests]


def poisson_arrivals(n: int, rate_per_s: float, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate_per_s, size=n))


def summarize(results: list[Result], makespan: float | None = None) -> dict:
    ok = [r for r in results if not r.error]
    lat = np.array([r.latency for r in ok]) if ok else np.zeros(1)
    span = makespan if makespan is not None else (max(r.finished for r in ok) - min(r.arrival for r in ok) if ok else 0)
    return {
        "requests": len(results), "completed": len(ok), "failed": len(results) - len(ok),
        "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
        "mean_latency_s": float(lat.mean()), "makespan_s": float(span),
        "traj_steps": int(sum(r.traj_steps for r in ok)),
        "traj_steps_per_s": float(sum(r.traj_steps for r in ok) / span) if span > 0 else math.nan,
    }
