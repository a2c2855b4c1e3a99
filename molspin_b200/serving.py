"""Serving form: continuous batching of field/orientation/system solves.

A request is one HSGeneral stochastic yield solve -- one radical-pair system
at one field orientation, as one RunSection step of the reference
(RunSection::Run -> TaskHSGeneral::RunLocal, main.cpp:651-678).  The engine
admits requests as they arrive, first-fit against a device-memory budget and
a number of slots.  Each admitted request runs on its own msgpu context (its
own CUDA stream; the budget it reserved is enforced by the context), and
worker threads drive the C ABI with the GIL released, so requests that
arrive while others run are admitted as soon as slots and memory free up
and their kernels overlap on the device.  Latency (arrival -> yields on the
host) is reported as p50/p99 beside throughput.

Contexts are pooled by request shape (dimension, trajectories, Krylov
dimension, steps): a finished request's context, with its device buffers,
its quartet-form and SpMM tuning, serves the next request of that shape, so
a steady stream allocates and frees no device memory (a cudaFree waits for
the whole device, i.e. for every other request's kernels).  Idle contexts
keep their reservation and are destroyed only when an admission needs the
memory.

Small systems share launches.  Requests below `pack_dim` (the batching
form's persistent route, D < 2048) that share a time grid and Krylov
dimension are admitted together, up to `pack_max` of them in one slot, and
run as one persistent launch of the batching form (msgpu_batch_*) on a
pooled batch whose device buffers are kept between packs
(msgpu_batch_clear).  A system's result in a batch does not depend on its
companions, and a small request solved alone also runs as a one-system
batch, so a packed result equals its solo run bit for bit.

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
    def __init__(self, device: int = 0, hbm_budget: int = 64 << 30, slots: int = 8, precision: str = "c64",
                 pack_dim: int = 2048, pack_max: int = 16):
        self.device = device
        self.budget = hbm_budget
        self.slots = slots
        self.precision = precision
        self.pack_dim = pack_dim    # requests below this dimension are packed (0: never)
        self.pack_max = pack_max    # requests per pack
        self._lock = threading.Condition()
        self._reserved = 0   # running requests plus idle pooled contexts
        self._running = 0    # slots in use (a pack takes one)
        self._inflight = 0   # requests running
        self._idle: dict[tuple, list[tuple[HSPropagatorB200, int]]] = {}  # shape -> [(context, reserved)]
        self._idle_batches: list[tuple[object, int]] = []                 # [(pooled batch, reserved)]
        self.packs = 0
        self.packed = 0
        self.max_concurrency = 0
        self.peak_reserved = 0
        self.contexts_created = 0
        self.contexts_reused = 0

    @staticmethod
    def shape(w: Workload) -> tuple:
        return (w.system.dim, w.M, w.krylov, w.steps)

    def packable(self, w: Workload) -> bool:
        return self.precision == "c64" and 0 < w.system.dim < self.pack_dim

    @staticmethod
    def pack_key(w: Workload) -> tuple:
        """Requests of one pack share the time grid and the Krylov dimension."""
        return (w.steps, w.dt, w.krylov)

    def _run(self, p: HSPropagatorB200, req: Request) -> np.ndarray:
        w = req.workload
        s = w.system
        F = s.trace_samples(w.M, w.seed)
        p.set_hamiltonian(*s.hamiltonian_csr())
        p.set_reaction(kappa=s.kappa())
        p.set_electron_pair(*s.electron_strides())
        p.set_observables([(op, rate) for _, op, rate in s.observables()])
        # every input is set on every request: a pooled context keeps the last one's
        if s.st_rate > 0.0:
            p.set_noise(s.st_rate, L.NOISE_PHILOX, req.seed)
        else:
            p.set_noise(0.0, L.NOISE_NONE)
        p.set_factors(F)
        p.propagate(w.times(), w.krylov, self.precision)
        _, ens = p.yields()
        return ens

    def solve(self, req: Request, budget: int = 0) -> np.ndarray:
        """One request on a context of its own (created and destroyed here;
        a one-system batch when it would be packed); returns the ensemble yields."""
        if self.packable(req.workload):
            ens, batch = self.solve_pack([req], None)
            batch.close()
            return ens[0]
        with HSPropagatorB200(self.device, budget) as p:
            return self._run(p, req)

    def solve_pack(self, reqs: list[Request], batch):
        """Requests of one pack key in one persistent launch on a pooled batch
        (a new one when batch is None); returns (ensemble yields per request,
        the batch to keep for the pool)."""
        from .batching import BatchB200
        if batch is None:
            batch = BatchB200(self.device)
        try:
            batch.clear()
            for q in reqs:
                w = q.workload
                batch.add(w.system, w.system.trace_samples(w.M, w.seed), q.seed)
            w0 = reqs[0].workload
            batch.run(w0.times(), w0.krylov)
            return [batch.yields(i)[1] for i in range(len(reqs))], batch
        except Exception:
            batch.close()
            raise

    def solve_pooled(self, req: Request, budget: int, ctx):
        """One request on a pooled context (a new one when ctx is None);
        returns (ensemble yields, the context to keep for the pool)."""
        if ctx is None:
            ctx = HSPropagatorB200(self.device, budget)
        try:
            return self._run(ctx, req), ctx
        except Exception:
            ctx.close()
            raise

    def _worker(self, req: Request, res: Result, t0: float, ctx):
        try:
            res.yields, ctx = self.solve_pooled(req, res.reserved, ctx)
        except Exception as e:  # noqa: BLE001 -- reported per request
            res.error = str(e)
            ctx = None
        res.finished = time.perf_counter() - t0
        with self._lock:
            if ctx is not None:
                self._idle.setdefault(self.shape(req.workload), []).append((ctx, res.reserved))
            else:
                self._reserved -= res.reserved
            self._running -= 1
            self._inflight -= 1
            self._lock.notify_all()

    def _pack_worker(self, reqs: list[Request], ress: list[Result], t0: float, batch, reserved: int):
        try:
            ens, batch = self.solve_pack(reqs, batch)
            for r, e in zip(ress, ens):
                r.yields = e
        except Exception as e:  # noqa: BLE001 -- reported per request
            for r in ress:
                r.error = str(e)
            batch = None
        fin = time.perf_counter() - t0
        for r in ress:
            r.finished = fin
        with self._lock:
            if batch is not None:
                self._idle_batches.append((batch, reserved))
            else:
                self._reserved -= reserved
            self._running -= 1
            self._inflight -= len(reqs)
            self._lock.notify_all()

    def _admit_pack(self, first: Request, waiting: list[Request], results: dict, now: float, t0: float,
                    threads: list) -> bool:
        """Admits `first` with the waiting requests of its pack key (called with
        the lock held and a slot free); False when not even `first` fits."""
        key = self.pack_key(first.workload)
        group = [q for q in waiting if self.packable(q.workload) and self.pack_key(q.workload) == key]
        group = group[:self.pack_max]
        batch, held = self._idle_batches.pop() if self._idle_batches else (None, 0)
        need = lambda g: max(held, sum(results[q.rid].reserved for q in g)) - held  # noqa: E731
        if self._reserved + need(group) > self.budget:
            evicted = self._evict(need(group))
            if evicted:
                self._lock.release()
                try:
                    for c, _ in evicted:
                        c.close()
                finally:
                    self._lock.acquire()
        while group and self._reserved + need(group) > self.budget:
            group.pop()
        if not group:
            if batch is not None:
                self._idle_batches.append((batch, held))
            return False
        extra = need(group)
        self._reserved += extra
        if batch is None:
            self.contexts_created += 1
        else:
            self.contexts_reused += 1
        for q in group:
            waiting.remove(q)
            results[q.rid].admitted = now
        self._running += 1
        self._inflight += len(group)
        self.packs += 1
        self.packed += len(group)
        self.max_concurrency = max(self.max_concurrency, self._inflight)
        self.peak_reserved = max(self.peak_reserved, self._reserved)
        th = threading.Thread(target=self._pack_worker,
                              args=(group, [results[q.rid] for q in group], t0, batch, held + extra), daemon=True)
        th.start()
        threads.append(th)
        return True

    def _evict(self, need: int) -> list[tuple[HSPropagatorB200, int]]:
        """Idle contexts to destroy (largest first) so that `need` more bytes fit;
        called with the lock held, the contexts are closed by the caller."""
        out = []
        pool = sorted(((r, k, i) for k, lst in self._idle.items() for i, (_, r) in enumerate(lst)), reverse=True)
        freed, take = 0, []
        for r, k, i in pool:
            if self._reserved - freed + need <= self.budget:
                break
            take.append((k, i))
            freed += r
        if self._reserved - freed + need > self.budget:
            return out  # evicting everything idle would not make room: wait for running requests
        for k, i in sorted(take, key=lambda x: -x[1]):
            out.append(self._idle[k].pop(i))
        for k in [k for k, lst in self._idle.items() if not lst]:
            del self._idle[k]
        self._reserved -= freed
        return out

    def close(self):
        """Destroys the idle pooled contexts and batches."""
        with self._lock:
            idle = [c for lst in self._idle.values() for c in lst] + self._idle_batches
            self._idle.clear()
            self._idle_batches = []
            self._reserved -= sum(r for _, r in idle)
        for ctx, _ in idle:
            ctx.close()

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
                # first fit: admit every waiting request that fits the free slots
                # and memory, on an idle pooled context of its shape if there is one
                k = 0
                while k < len(waiting) and self._running < self.slots:
                    req = waiting[k]
                    res = results[req.rid]
                    if self.packable(req.workload):
                        if not self._admit_pack(req, waiting, results, now, t0, threads):
                            k += 1
                        continue
                    ctx = None
                    pooled = self._idle.get(self.shape(req.workload))
                    if pooled:
                        ctx, res.reserved = pooled.pop()
                        self.contexts_reused += 1
                    else:
                        if self._reserved + res.reserved > self.budget:
                            evicted = self._evict(res.reserved)
                            if evicted:
                                self._lock.release()
                                try:
                                    for c, _ in evicted:
                                        c.close()
                                finally:
                                    self._lock.acquire()
                        if self._reserved + res.reserved > self.budget:
                            k += 1
                            continue
                        self._reserved += res.reserved
                        self.contexts_created += 1
                    waiting.pop(k)
                    self._running += 1
                    self._inflight += 1
                    self.max_concurrency = max(self.max_concurrency, self._inflight)
                    self.peak_reserved = max(self.peak_reserved, self._reserved)
                    res.admitted = now
                    th = threading.Thread(target=self._worker, args=(req, res, t0, ctx), daemon=True)
                    th.start()
                    threads.append(th)
                if i >= len(order) and not waiting and self._running == 0:
                    break
                timeout = None
                if realtime and i < len(order):
                    timeout = max(0.0, order[i].arrival - (time.perf_counter() - t0))
                self._lock.wait(timeout=timeout if timeout is not None else 1.0)
        for th in threads:
            th.join()
        self.close()
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
