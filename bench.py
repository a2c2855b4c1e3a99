"""Benchmark: stochastic HSGeneral trajectory-steps/s on B200.

Workload (the precision-form configuration): radical pair with 2 electrons and
12 spin-1/2 nuclei (8 on A, 4 on B), D = 16384, anisotropic hyperfine tensors
(seed 1), B = 50 uT in a random direction, 1024 trace-sampled trajectories,
Krylov dimension 20, dt = 0.5 ns, symmetric recombination k = 1/us; bulk
complex64 with FP64 reductions (Lanczos, expm, yield sums).  Synthetic,
seeded inputs of the configuration's shapes.

One bench step = `--chunk` time steps of the whole 1024-trajectory block
(one msgpu_run call).  value = trajectory-steps per second over the K timed
steps (max over ranks; ranks hold independent trajectory blocks: weak
scaling, no collective in the data path).  Inputs (the 128 MiB state and the
2.6 GiB Krylov basis) are larger than L2, so no L2 flush is needed.

--impl reference times the CPU restatement of the reference algorithm
(oracle/, complex128 Arnoldi as in SpinSpace::KrylovExpmGeneral) on all host
cores on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--chunk", type=int, default=50, help="time steps per bench step")
    ap.add_argument("--traj", type=int, default=1024)
    ap.add_argument("--plain-steps", type=int, default=50,
                    help="time steps of the complex128 comparison run (one bench step)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-segments", action="store_true",
                    help="precision line only (no dense, batching and serving segments)")
    ap.add_argument("--workload", default="precision", choices=["precision", "plain", "dense", "batching", "serving"],
                    help="precision (default line): D=16384 complex64; plain: D=64 complex128; dense: D=1024 "
                         "tensor-core propagator; batching: 64 uneven systems; serving: a request stream")
    ap.add_argument("--requests", type=int, default=40, help="serving: requests in the stream")
    ap.add_argument("--rate", type=float, default=4.0, help="serving: Poisson arrival rate (requests/s)")
    ap.add_argument("--pack-dim", type=int, default=2048,
                    help="serving: requests below this dimension share batch launches (0: one context each)")
    ap.add_argument("--precision", default=None, help="dense: bf16x3 | bf16x6 | int8x4")
    ap.add_argument("--spmm-variant", type=int, default=-1,
                    help="precision form: -1 autotuned SpMM variant (default), k >= 0 force variant k")
    ap.add_argument("--combine-tile", type=int, default=0,
                    help="precision form: quartets per CTA of the combine (MSGPU_OPT_COMBINE_TILE; 0 default)")
    ap.add_argument("--traj-groups", type=int, default=0,
                    help="precision form: trajectory groups of the step (MSGPU_OPT_TRAJ_GROUPS; 0 default)")
    ap.add_argument("--lanczos-cluster", type=int, default=0,
                    help="precision form: 0 four-kernel Lanczos iteration (default); -1, 1, 2, 4, 8, 16 the "
                         "cluster-resident recurrence (MSGPU_OPT_LANCZOS_CLUSTER)")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for name, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(name)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def _dist():
    from molspin_b200 import ranks
    return ranks.init()


def _max_over_ranks(x: float, world: int) -> float:
    from molspin_b200 import ranks
    return ranks.max_over_ranks(x, world)


def _barrier(world: int):
    from molspin_b200 import ranks
    ranks.barrier(world)


# Bounded CPU samples: about 10 s of work each (the oracle's rate per core is
# fixed, so the trajectory count follows the core count).
CPU_SAMPLE_STEPS = 128  # precision workload: 2 trajectories per core x 128 steps

# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one SpMM launch
# from an ncu capture, by (D, trajectories per launch): 1024 trajectories (one
# group): 138.4 MB + 105.5 MB; 512 (one of two groups): 73.9 MB + 43.6 MB
TRAFFIC_SPMM = {(16384, 1024): 243.9e6, (16384, 512): 117.5e6}


def _oracle_inputs(w, traj: int, steps: int):
    """Inputs of a CPU sample built by the oracle alone (trace samples, sparse Kronecker H,
    pair observables, time grid), so that the CPU legs never load the product library."""
    from oracle import density as den
    from oracle import pyoracle as orc
    from molspin_b200 import systems as S
    F = orc.trace_samples(float(w.seed), S.SINGLET, w.system.dim // 4, traj)
    times = orc.time_grid(steps * w.dt, w.dt)
    obs = [(den.pair_operator_csr(op, w.system), rate) for _, op, rate in w.system.observables()]
    return F, times, obs, den.sparse_hamiltonian(w.system)


def cpu_reference(w, sample_traj: int, sample_steps: int, threads: int) -> dict:
    """The CPU restatement (complex128 Arnoldi/MGS, per-column Krylov) on a bounded sample."""
    from oracle import pyoracle as orc
    F, times, obs, Hc = _oracle_inputs(w, sample_traj, sample_steps)
    orc.hs_stochastic(Hc, F[:, :threads], times[:2], obs, kappa=w.system.kappa(), krylov=w.krylov,
                      nthreads=threads)  # warm-up
    t0 = time.perf_counter()
    orc.hs_stochastic(Hc, F, times, obs, kappa=w.system.kappa(), krylov=w.krylov, nthreads=threads)
    el = time.perf_counter() - t0
    return {"value": sample_traj * sample_steps / el, "unit": "traj-steps/s", "cores": threads, "kind": "port",
            "sample": f"{sample_traj} trajectories x {sample_steps} steps of the D={w.system.dim} m={w.krylov} "
                      f"workload (complex128 Arnoldi, {el:.1f} s)"}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from molspin_b200 import systems as S
    w = S.precision_large(M=args.traj, steps=args.chunk)
    threads = os.cpu_count() or 1
    traj = 2 * threads
    for _ in range(max(0, min(args.warmup, 1))):
        cpu_reference(w, threads, 1, threads)
    vals = []
    for _ in range(max(1, min(args.steps, 3))):
        vals.append(cpu_reference(w, traj, CPU_SAMPLE_STEPS, threads))
    v = sum(x["value"] for x in vals) / len(vals)
    line = {
        "impl": "reference", "metric": "SSE traj-steps/s (stochastic HSGeneral, Krylov m=20, D=16384)",
        "value": v, "unit": "traj-steps/s", "n_gpus": world, "steps": len(vals), "warmup": args.warmup,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic (seeded)",
        "config": {"workload": w.name, "trajectories": args.traj, "dim": w.system.dim, "krylov": w.krylov},
        "cpu_baseline": {**vals[-1], "value": v},
        "e2e": {"value": v, "unit": "traj-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference binary not buildable here (Armadillo absent): CPU restatement of its algorithm, all cores",
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    import numpy as np
    import torch

    from molspin_b200 import _lib as L
    from molspin_b200 import hsgeneral as hs
    from molspin_b200 import ranks
    from molspin_b200 import systems as S

    world, rank, local = _dist()
    M, chunk, K, W = args.traj, args.chunk, args.steps, args.warmup
    w = S.precision_large(M=M, steps=chunk)
    sysm = w.system
    D = sysm.dim
    rowptr, col, val = sysm.hamiltonian_csr()
    F = sysm.trace_samples(M, ranks.block_seed(w.seed, rank))
    obs = [(op, rate) for _, op, rate in sysm.observables()]
    times = S.time_grid(chunk * w.dt, w.dt)
    stream = torch.cuda.current_stream()

    p = hs.HSPropagatorB200(local)
    L.lib.msgpu_set_stream(p.ctx, stream.cuda_stream)
    if args.spmm_variant >= 0:
        p.set_option(L.OPT_SPMM_VARIANT, args.spmm_variant)
    if args.lanczos_cluster:
        p.set_option(L.OPT_LANCZOS_CLUSTER, args.lanczos_cluster)
    if args.combine_tile:
        p.set_option(L.OPT_COMBINE_TILE, args.combine_tile)
    if args.traj_groups:
        p.set_option(L.OPT_TRAJ_GROUPS, args.traj_groups)
    p.set_hamiltonian(rowptr, col, val)
    p.set_reaction(kappa=sysm.kappa())
    p.set_electron_pair(*sysm.electron_strides())
    p.set_observables(obs)
    p.set_factors(F)
    groups = int(p.get_option(L.OPT_TRAJ_GROUPS))  # trajectory groups of the step (one SpMM launch each)

    def bench_step(first: bool, k: int):
        p.propagate(times, w.krylov, "c64", step_offset=k * chunk, accumulate=not first)

    # warm-up
    for k in range(W):
        bench_step(k == 0, k)
    _barrier(world)
    launches0 = p.launch_count()
    p.profile(2)  # sampled: every launch of every 32nd time step
    clocks = ClockSampler(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    _barrier(world)
    ev0.record(stream)
    for k in range(K):
        bench_step(False, W + k)
    ev1.record(stream)
    _barrier(world)
    clk = clocks.stop()
    el_ms = ev0.elapsed_time(ev1)
    apply_ms, apply_n = p.profile_read(L.KC_APPLY)
    orth_ms, orth_n = p.profile_read(L.KC_ORTH)
    red_ms, red_n = p.profile_read(L.KC_REDUCE)
    comb_ms, comb_n = p.profile_read(L.KC_COMBINE)
    fused_ms, fused_n = p.profile_read(L.KC_LANCZOS)
    p.profile(False)
    launches = p.launch_count() - launches0
    el_max = _max_over_ranks(el_ms, world)
    value = ranks.aggregate(M * chunk * K, world, el_max / 1e3)

    # roofline of the dominant kernel (Lanczos SpMM): algorithmic bytes per
    # launch = read the block's Krylov vector once + write H v once (D*M*8 each)
    # + the CSR Hamiltonian (nnz * (8 + 4) + 4 (D+1)).
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_kind = "measured" if "hbm_gbs" in peaks else "fallback"
    width = M // groups  # trajectories of one SpMM launch
    alg_bytes = 2 * D * width * 8 + len(col) * 12 + 4 * (D + 1)
    traffic = TRAFFIC_SPMM.get((D, width))
    apply_avg_s = apply_ms / max(1, apply_n) / 1e3
    achieved = alg_bytes / apply_avg_s / 1e9 if apply_n else None
    # the whole time step against HBM: m SpMMs, m-1 updates (4 vectors each) and
    # the combine ((m + 2) vectors); expm, reductions and yields are negligible
    # the minimal fused Krylov traffic per time step, (4m+1) D c per trajectory (c = 8 B), and the
    # traffic of the kernels as they are split here (m SpMMs, m-1 four-vector updates, the combine)
    m_k = w.krylov
    step_bytes = (4 * m_k + 1) * D * 8 * M
    step_bytes_split = m_k * groups * alg_bytes + (m_k - 1) * 4 * D * M * 8 + (m_k + 2) * D * M * 8
    step_s = el_max / 1e3 / (K * chunk)

    # plain complex128 path (reference-faithful Arnoldi) on a short segment,
    # and the singlet-yield deviation of the complex64 form from it
    Fp = F[:, :M]
    plain_steps = args.plain_steps
    plain_value, yerr = None, None
    if plain_steps > 0:
        tp = S.time_grid(plain_steps * w.dt, w.dt)
        p.set_factors(Fp)
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        p.propagate(tp, w.krylov, "c128")  # warm
        p.set_factors(Fp)
        t0.record(stream)
        p.propagate(tp, w.krylov, "c128")
        t1.record(stream)
        torch.cuda.synchronize()
        plain_value = M * plain_steps / (t0.elapsed_time(t1) / 1e3)
        _, ens128 = p.yields()
        p.set_factors(Fp)
        p.propagate(tp, w.krylov, "c64")
        _, ens64 = p.yields()
        yerr = abs(ens64[0] - ens128[0]) / abs(ens128[0])

    # end to end through the public API with host buffers: every step uploads
    # the factor block from pinned host memory, runs, and reads the yields back
    e2e = None
    if not args.no_e2e:
        pinned = torch.empty((M, D), dtype=torch.complex128, pin_memory=True)
        pinned.numpy()[:] = F.T
        per = np.zeros((M, len(obs)))
        ens = np.zeros(len(obs))
        E = max(1, min(K, 3))
        _barrier(world)
        t_0 = time.perf_counter()
        for k in range(E):
            rc = L.lib.msgpu_upload_factors(p.ctx, D, M, L.C.cast(pinned.data_ptr(), L.C.POINTER(L.C.c_double)))
            assert rc == 0, L.lib.msgpu_last_error(p.ctx)
            p.propagate(times, w.krylov, "c64", step_offset=k * chunk)
            hs._check(p.ctx, L.lib.msgpu_fetch_yields(p.ctx, L.dptr(per), L.dptr(ens)))
        _barrier(world)
        el_e2e = _max_over_ranks(time.perf_counter() - t_0, world)
        e2e = {"value": world * M * chunk * E / el_e2e, "unit": "traj-steps/s",
               "h2d_bytes_per_step": D * M * 16, "d2h_bytes_per_step": per.nbytes + ens.nbytes + len(times) * len(obs) * 8,
               "steps": E}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        cpu = cpu_reference(w, 2 * threads, CPU_SAMPLE_STEPS, threads)

    spmm = p.spmm_choice()  # what the tuner picked (or the forced variant)
    p.close()
    segments = {} if args.no_segments else run_segments(args)
    line = None
    if rank == 0:
        line = {
            "metric": "SSE traj-steps/s (stochastic HSGeneral, Krylov m=20, D=16384)",
            "value": value, "unit": "traj-steps/s", "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": el_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c64 (FP64 reductions/expm/sums)", "data": "synthetic (seeded)",
            "config": {"workload": w.name, "trajectories_per_gpu": M, "dim": D, "nnz": int(len(col)),
                       "krylov": w.krylov, "dt_ns": w.dt, "time_steps_per_bench_step": chunk,
                       "l2": "inputs larger than L2 (no flush)", "recurrence": "lanczos", "trajectory_groups": groups,
                       "spmm": spmm, "parallelism": f"independent trajectory blocks x{world}"},
            "roofline": {"bound": "hbm", "kernel": "quartet SpMM (k_lanczos_apply_*, autotuned variant)", "achieved": achieved, "peak": hbm_peak,
                         "unit": "GB/s", "frac": (achieved / hbm_peak) if achieved else None, "traffic": traffic,
                         "peak_kind": peak_kind, "alg_bytes_per_launch": alg_bytes,
                         "avg_launch_ms": apply_avg_s * 1e3, "launches_timed": apply_n,
                         "timing": "CUDA events around every launch of every 32nd time step (sampled)",
                         "share_of_step": apply_avg_s * 1e3 * w.krylov * groups * chunk * K / el_ms if el_ms else None,
                         "trajectories_per_launch": width},
            "step_roofline": {"bound": "hbm", "alg_bytes_per_time_step": step_bytes,
                              "alg_bytes": "(4m+1) D c per trajectory: the minimal fused Krylov traffic",
                              "time_step_ms": step_s * 1e3,
                              "achieved": step_bytes / step_s / 1e9, "peak": hbm_peak, "unit": "GB/s",
                              "frac": step_bytes / step_s / 1e9 / hbm_peak, "peak_kind": peak_kind,
                              "split_kernel_bytes_per_time_step": step_bytes_split,
                              "split_kernel_frac": step_bytes_split / step_s / 1e9 / hbm_peak},
            "kernel_avg_ms": {"apply": apply_ms / max(1, apply_n), "update": orth_ms / max(1, orth_n),
                              "reduce": red_ms / max(1, red_n),
                              "combine": comb_ms / max(1, comb_n),
                              **({"lanczos_cluster_resident": fused_ms / fused_n} if fused_n else {})},
            "lanczos": "cluster-resident recurrence" if fused_n else "SpMM + update + reductions per iteration",
            "plain_c128": {"value": plain_value, "unit": "traj-steps/s", "steps": plain_steps,
                           "speedup_of_c64": (value / world / plain_value) if plain_value else None},
            "yield_rel_err_c64_vs_c128": yerr,
            "clocks": clk,
            "e2e": e2e,
            "gpu_launches": launches,
            "cpu_baseline": cpu,
            "segments": segments,
        }
    return rank, line


def run_segments(args) -> dict:
    """Short driver-clocked runs of the other configurations after the contract line (each with
    its own clocks, launch count and roofline where one applies): the dense tensor-core form
    (config 4 shape, 1000 timed steps), the batching form (the 64-system batch, 200 timed steps)
    and a serving stream below saturation (12 requests of the serving mix at 0.25 requests/s)."""
    import copy
    out = {}
    for name, fn, kw in (("dense", run_dense, dict(chunk=500, steps=2, warmup=3)),
                         ("batching", run_batching, dict(chunk=100, steps=2, warmup=3)),
                         ("serving", run_serving, dict(requests=12, rate=0.25))):
        a = copy.copy(args)
        a.no_cpu = True
        a.traj = 1024  # the runners' own defaults
        for k, v in kw.items():
            setattr(a, k, v)
        _, line = fn(a)
        if line is not None:
            line.pop("cpu_baseline", None)
            out[name] = line
    return out


def _peaks() -> dict:
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def _propagator(system, local: int, stream=None):
    from molspin_b200 import _lib as L
    from molspin_b200 import hsgeneral as hs
    p = hs.HSPropagatorB200(local)
    if stream is not None:
        L.lib.msgpu_set_stream(p.ctx, stream.cuda_stream)
    p.set_hamiltonian(*system.hamiltonian_csr())
    p.set_reaction(kappa=system.kappa())
    p.set_electron_pair(*system.electron_strides())
    p.set_observables([(op, rate) for _, op, rate in system.observables()])
    return p


def _timed(world, stream, fn, W, K):
    """W untimed calls, then K calls between barriers; device time (ms) max over ranks."""
    import torch
    for k in range(W):
        fn(k)
    _barrier(world)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    ev0.record(stream)
    for k in range(K):
        fn(W + k)
    ev1.record(stream)
    _barrier(world)
    clk = clocks.stop()
    return _max_over_ranks(ev0.elapsed_time(ev1), world), clk


def _e2e(p, world, F, times, krylov, precision, propagator, E):
    """Through the public API with host buffers: upload the factor block from
    pinned memory, run, read the yields back, every step."""
    import numpy as np
    import torch
    from molspin_b200 import _lib as L
    from molspin_b200 import hsgeneral as hs
    D, M = F.shape
    pinned = torch.empty((M, D), dtype=torch.complex128, pin_memory=True)
    pinned.numpy()[:] = F.T
    per = np.zeros((M, p.nobs))
    ens = np.zeros(p.nobs)
    _barrier(world)
    t0 = time.perf_counter()
    for k in range(E):
        hs._check(p.ctx, L.lib.msgpu_upload_factors(p.ctx, D, M, L.C.cast(pinned.data_ptr(), L.C.POINTER(L.C.c_double))))
        p.propagate(times, krylov, precision, step_offset=k * (len(times) - 1), propagator=propagator)
        hs._check(p.ctx, L.lib.msgpu_fetch_yields(p.ctx, L.dptr(per), L.dptr(ens)))
    _barrier(world)
    el = _max_over_ranks(time.perf_counter() - t0, world)
    return {"value": world * M * (len(times) - 1) * E / el, "unit": "traj-steps/s", "h2d_bytes_per_step": D * M * 16,
            "d2h_bytes_per_step": per.nbytes + ens.nbytes + len(times) * p.nobs * 8, "steps": E}


def _cpu_port(w, traj: int, steps: int, method: int = 0) -> dict:
    """The oracle (CPU restatement of the reference algorithm) on all host cores."""
    from oracle import pyoracle as orc
    threads = os.cpu_count() or 1
    F, times, obs, Hc = _oracle_inputs(w, traj, steps)
    t0 = time.perf_counter()
    orc.hs_stochastic(Hc, F, times, obs, kappa=w.system.kappa(), krylov=w.krylov, method=method, nthreads=threads)
    el = time.perf_counter() - t0
    return {"value": traj * steps / el, "unit": "traj-steps/s", "cores": threads, "kind": "port",
            "sample": f"{traj} trajectories x {steps} steps of {w.name} ({el:.1f} s)"}


def _emit(rank, line):
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_plain(args):
    """Plain complex128 form on the CPU-runnable configuration (D=64, 256
    trajectories, m=16, dt=1 ns): the whole time loop runs resident on the device."""
    import torch
    from molspin_b200 import systems as S
    world, rank, local = _dist()
    w = S.plain_small()
    chunk = args.chunk if args.chunk != 50 else 1000
    F = w.system.trace_samples(w.M, w.seed + rank)
    times = S.time_grid(chunk * w.dt, w.dt)
    stream = torch.cuda.current_stream()
    p = _propagator(w.system, local, stream)
    p.set_factors(F)
    l0 = [0]

    def step(k):
        if k == args.warmup:
            l0[0] = p.launch_count()
        p.propagate(times, w.krylov, "c128", step_offset=k * chunk, accumulate=k > 0)
    el, clk = _timed(world, stream, step, args.warmup, args.steps)
    launches = p.launch_count() - l0[0]
    e2e = None if args.no_e2e else _e2e(p, world, F, times, w.krylov, "c128", "krylov", max(1, min(args.steps, 3)))
    p.close()
    cpu = _cpu_port(w, w.M, w.steps) if rank == 0 and world == 1 and not args.no_cpu else None  # the whole workload
    return rank, ({
        "metric": "SSE traj-steps/s (plain complex128, D=64, m=16)", "value": world * w.M * chunk * args.steps / (el / 1e3),
        "unit": "traj-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": el / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c128", "data": "synthetic (seeded)",
        "config": {"workload": w.name, "trajectories_per_gpu": w.M, "time_steps_per_bench_step": chunk,
                   "form": "resident (one launch per bench step)", "l2": "state resident on chip (no flush)"},
        "roofline": None, "clocks": clk, "e2e": e2e, "gpu_launches": launches, "cpu_baseline": cpu})


def run_dense(args):
    """Dense tensor-core form: D=1024 time-independent H, U = exp(-iH dt) in
    FP64 once, then a split-BF16 tcgen05 GEMM over the 4096-trajectory block."""
    import numpy as np
    import torch
    from molspin_b200 import _lib as L
    from molspin_b200 import systems as S
    world, rank, local = _dist()
    prec = args.precision or "bf16x3"
    M = args.traj if args.traj != 1024 else 4096
    chunk = args.chunk if args.chunk != 50 else 500
    w = S.dense_tc(M=M, steps=chunk)
    D = w.system.dim
    F = w.system.trace_samples(M, w.seed + rank)
    times = S.time_grid(chunk * w.dt, w.dt)
    stream = torch.cuda.current_stream()
    p = _propagator(w.system, local, stream)
    p.set_factors(F)
    p.propagate(times[:3], w.krylov, prec, propagator="dense")  # U precompute + buffers
    p.set_factors(F)
    l0 = [0]

    def step(k):
        if k == args.warmup:
            l0[0] = p.launch_count()
            p.profile(2)  # sampled: every 8th GEMM
        p.propagate(times, w.krylov, prec, step_offset=k * chunk, accumulate=k > 0, propagator="dense")
    el, clk = _timed(world, stream, step, args.warmup, args.steps)
    launches = p.launch_count() - l0[0]
    gms, gn = p.profile_read(6)
    p.profile(False)
    nprod = {"bf16x3": 3, "bf16x6": 6, "int8x4": 10}[prec]
    Dp = (2 * D + 127) // 128 * 128
    flops = 2.0 * Dp * Dp * M * nprod
    achieved = flops / (gms / gn / 1e3) / 1e12 if gn else None
    peaks = _peaks()
    peak = float(peaks.get("bf16_tflops_sustained", 1400.0))
    # int8 products: the peak file holds no int8 figure.  cuBLASLt int8 (torch._int_mm) against
    # cuBLAS BF16 on this GPU type, both 8192^3 bursts in one process, measured 2907.8 TOP/s
    # against 1642.6 TFLOP/s: the int8 peak is the BF16 figure times that ratio
    peak_note = "measured sustained BF16" if "bf16_tflops_sustained" in peaks else "fallback BF16"
    if prec == "int8x4":
        peak *= 2907.8 / 1642.6
        peak_note = "1.77 x the " + peak_note + " (measured cuBLASLt int8 / cuBLAS BF16 ratio)"
    # DRAM bytes per GEMM launch from one ncu capture (bf16x3, D=1024, M=4096:
    # 55.1 MB read + 6.8 MB written; the output stays partly in L2)
    traffic = 61.9e6 if (D, M, prec) == (1024, 4096, "bf16x3") else None
    # accuracy against the complex128 Krylov path on a 256-trajectory subset
    sub = min(256, M)
    Fs = np.ascontiguousarray(F[:, :sub])
    ts = S.time_grid(200 * w.dt, w.dt)
    p2 = _propagator(w.system, local, stream)
    p2.set_factors(Fs)
    p2.propagate(ts, w.krylov, "c128")
    per128, ens128 = p2.yields()
    p2.set_factors(Fs)
    p2.propagate(ts, w.krylov, prec, propagator="dense")
    perd, ensd = p2.yields()
    p2.set_option(L.OPT_DENSE_RENORMALIZE, 0)
    p2.set_factors(Fs)
    p2.propagate(ts, w.krylov, prec, propagator="dense")
    raw = p2.get_factors()
    exact = np.sum(np.abs(Fs) ** 2, axis=0) * np.exp(-2.0 * w.system.kappa() * ts[-1])
    drift = float(np.max(np.abs(np.sum(np.abs(raw) ** 2, axis=0) / exact - 1.0)) / 200)
    p2.close()
    e2e = None if args.no_e2e else _e2e(p, world, F, times, w.krylov, prec, "dense", max(1, min(args.steps, 3)))
    p.close()
    # the reference has no dense propagator: its CPU path is the Krylov step
    cpu = _cpu_port(w, 8 * (os.cpu_count() or 1), 600) if rank == 0 and world == 1 and not args.no_cpu else None
    return rank, ({
        "metric": "SSE traj-steps/s (dense tensor-core propagator, D=1024)",
        "value": world * M * chunk * args.steps / (el / 1e3), "unit": "traj-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": ("int8x4: four int8 slices, exact int32 accumulation, FP64 state" if prec == "int8x4"
                  else f"{prec} split BF16, FP32 accumulate"),
        "data": "synthetic (seeded)",
        "config": {"workload": w.name, "trajectories_per_gpu": M, "time_steps_per_bench_step": chunk,
                   "renormalize": "exact Haberkorn survival", "l2": "state 2 x 33 MiB + U 16-24 MiB per step"},
        "roofline": {"bound": "tensor", "kernel": "k_dense_gemm_i8" if prec == "int8x4" else "k_dense_gemm",
                     "achieved": achieved, "peak": peak,
                     "unit": "TOP/s" if prec == "int8x4" else "TFLOP/s", "frac": achieved / peak if achieved else None,
                     "traffic": traffic, "peak_kind": peak_note,
                     "flops_per_launch": flops, "avg_launch_ms": gms / gn if gn else None,
                     # the complex product itself, 8 D^2 flops per trajectory (one complex MAC = 8
                     # real flops), against the split products the tensor cores execute
                     "algorithmic_flops_per_launch": 8.0 * D * D * M,
                     "algorithmic_tflops": (8.0 * D * D * M) / (gms / gn / 1e3) / 1e12 if gn else None,
                     "launches_timed": gn, "timing": "CUDA events around every 8th GEMM (sampled)",
                     "share_of_step": (gms / gn) * chunk * args.steps / el if gn and el else None},
        "accuracy_vs_c128_200_steps": {
            "traj_yield_rel": float(np.max(np.abs(perd - per128)) / np.max(np.abs(per128))),
            "ensemble_yield_rel": float(np.max(np.abs(ensd - ens128) / np.abs(ens128))),
            "norm_drift_per_step_unrenormalised": drift},
        "clocks": clk, "e2e": e2e, "gpu_launches": launches, "cpu_baseline": cpu})


def run_batching(args):
    """Batching form: 64 systems of uneven dimension (64..9216) and uneven
    trajectory counts (64..1024) advanced in one persistent graph-replayed launch."""
    import torch
    from molspin_b200 import batching as B
    from molspin_b200 import systems as S
    world, rank, local = _dist()
    chunk = args.chunk if args.chunk != 50 else 100
    ws = S.batching_systems(steps=chunk)
    times = S.time_grid(chunk * 1.0, 1.0)
    stream = torch.cuda.current_stream()
    bt = B.BatchB200(local)
    for i, w in enumerate(ws):
        bt.add(w.system, w.system.trace_samples(w.M, w.seed + rank), 1000 + i)
    t0 = time.perf_counter()
    bt.tune(times[:6], 16)
    tune_s = time.perf_counter() - t0
    ms = []
    l0 = [0]

    def step(k):
        if k == args.warmup:
            l0[0] = bt.launch_count()
        bt.run(times, 16, step_offset=k * chunk, accumulate=k > 0)
        ms.append(bt.stats()["last_run_ms"])
    _, clk = _timed(world, stream, step, args.warmup, args.steps)
    launches = bt.launch_count() - l0[0]
    # the batch runs on its own streams: the library's time of each run (device
    # events around the graph replay, or the wall time of the whole run when
    # large systems take the streamed path on further streams)
    el = _max_over_ranks(sum(ms[args.warmup:]), world)
    st = bt.stats()
    Mtot = sum(w.M for w in ws)
    # per-system routes and, for the streamed systems, the SpMM each one's tuner picked
    infos = [bt.system_info(i) for i in range(len(ws))]
    picks = {}
    for i, inf in enumerate(infos):
        if inf["streamed"]:
            key = f"variant {inf['spmm_variant']} tile {inf['spmm_tile']} groups {inf['traj_groups']}"
            picks.setdefault(key, []).append(ws[i].system.dim)
    bt.close()
    # whole-batch HBM roofline with the minimal fused Krylov traffic (4m+1) D c per traj-step
    # (complex64, c = 8 B); the persistent kernel keeps small systems on chip, so this is the
    # bound the streamed large systems face
    bytes_per_step = sum((4 * 16 + 1) * w.system.dim * 8 * w.M for w in ws)
    peaks = _peaks()
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    achieved = bytes_per_step * chunk * args.steps / (el / 1e3) / 1e9 if el else None
    return rank, ({
        "metric": "SSE traj-steps/s (batching form, 64 uneven systems)",
        "value": world * Mtot * chunk * args.steps / (el / 1e3), "unit": "traj-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c64 (FP64 reductions/expm/sums)", "data": "synthetic (seeded)",
        "config": {"workload": "64 radical pairs, 4-10 nuclei (0-2 spin-1), dims 64-9216, M 64-1024, dt=1 ns",
                   "trajectories_per_gpu": Mtot, "time_steps_per_bench_step": chunk, "team_threshold": st["team_threshold"],
                   "ctas_per_sm": st["ctas_per_sm"], "tune_s": tune_s},
        "roofline": {"bound": "hbm", "kernel": "whole batch ((4m+1) D c bytes per traj-step)",
                     "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm if achieved else None,
                     "traffic": None, "peak_kind": "measured" if "hbm_gbs" in peaks else "fallback"},
        "clocks": clk, "e2e": None, "gpu_launches": launches,
        "routes": {"persistent": sum(not i["streamed"] for i in infos), "streamed": sum(i["streamed"] for i in infos),
                   "streamed_spmm_picks": {k: sorted(v) for k, v in picks.items()}},
        "launch_note": "per bench step: one graph replay of the persistent k_batch launch (systems below D=2048) "
                       "plus the streamed path's kernels for the larger systems", "cpu_baseline": None})


def run_serving(args):
    """Serving form: a Poisson request stream (6-14 nuclei, D=256..65536,
    256 trajectories, ST dephasing, 3000 steps) admitted under a device-memory budget."""
    from molspin_b200 import serving as SV
    from molspin_b200 import systems as S
    world, rank, local = _dist()
    import torch
    grid = S.sphere_grid(200)
    arr = SV.poisson_arrivals(args.requests, args.rate, seed=5 + rank)
    reqs = [SV.Request(i, float(arr[i]), S.serving_request(i + 100000 * rank, grid), seed=7000 + i)
            for i in range(args.requests)]
    pack_dim = getattr(args, "pack_dim", 2048)
    eng = SV.ServingEngine(local, hbm_budget=120 << 30, slots=8, pack_dim=pack_dim)
    clocks = ClockSampler(local)
    clocks.start()
    _barrier(world)
    t0 = time.perf_counter()
    res = eng.serve(reqs)
    torch.cuda.synchronize()
    el = _max_over_ranks(time.perf_counter() - t0, world)
    clk = clocks.stop()
    s = SV.summarize(res)
    # HBM roofline of the whole stream with the minimal fused Krylov traffic (4m+1) D c per
    # traj-step (complex64, c = 8 B)
    total_bytes = sum((4 * r.workload.krylov + 1) * r.workload.system.dim * 8 * r.workload.M * r.workload.steps
                      for r in reqs) * world
    peaks = _peaks()
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    achieved = total_bytes / el / 1e9
    return rank, ({
        "metric": "SSE traj-steps/s (serving form, continuous batching)", "value": world * s["traj_steps"] / el,
        "unit": "traj-steps/s", "n_gpus": world, "steps": 1, "warmup": 0, "ms_per_step": el * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64 (FP64 reductions/expm/sums)",
        "data": "synthetic (seeded)",
        "config": {"workload": f"{args.requests} requests, Poisson {args.rate}/s, 6-14 nuclei, M=256, 3000 steps",
                   "slots": 8, "hbm_budget_gib": 120, "pack_dim": pack_dim},
        "latency_s": {"p50": s["p50_latency_s"], "p99": s["p99_latency_s"], "mean": s["mean_latency_s"]},
        "completed": s["completed"], "failed": s["failed"], "max_concurrency": eng.max_concurrency,
        "contexts": {"created": eng.contexts_created, "reused": eng.contexts_reused},
        "packs": {"launches": eng.packs, "requests": eng.packed},
        "peak_reserved_gib": eng.peak_reserved / 2 ** 30,
        "roofline": {"bound": "hbm", "kernel": "whole stream ((4m+1) D c bytes per traj-step)", "achieved": achieved,
                     "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "traffic": None,
                     "peak_kind": "measured" if "hbm_gbs" in peaks else "fallback"},
        "clocks": clk, "e2e": None,
        "gpu_launches": None, "cpu_baseline": None})


def main():
    args = _args()
    if args.impl == "reference":
        run_reference(args)
    else:
        runner = {"plain": run_plain, "dense": run_dense, "batching": run_batching, "serving": run_serving,
                  "precision": run_ours}[args.workload]
        rank, line = runner(args)
        _emit(rank, line)
    from molspin_b200 import ranks
    ranks.finish(int(os.environ.get("WORLD_SIZE", "1")))


if __name__ == "__main__":
    main()
