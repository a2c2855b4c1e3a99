"""GPU parity of the dense tensor-core form (MSGPU_PROP_DENSE).

U = exp((-iH - K) dt) is built once in FP64 on the device and applied to the
whole trajectory block each step as a real-form complex GEMM on tcgen05, with
both operands split into BF16 parts (bf16x3: 2 parts, 3 products; bf16x6: 3
parts, 6 products) and FP32 accumulation in tensor memory, or cut into four
int8 slices with exact int32 accumulation and an FP64 state (int8x4).  The
oracle is the
same trajectory algorithm with an FP64 expm propagator (method=1), itself
pinned against the Krylov oracle to 1e-12.

Tolerances are stated per test.  The FP32 accumulation of the tensor cores
rounds towards zero and shrinks the state by about 1e-6 (bf16x3) and 5e-7
(bf16x6) per step at D=1024 (the split corrections accumulate separately, and
bf16x6 spreads the hi x hi product over three K ranges); with symmetric
recombination the exact survival is known, so the renormalised run (the
default) removes the uniform part and the yields carry only the non-uniform
remainder.
"""
import numpy as np
import pytest

from molspin_b200 import _lib as L
from molspin_b200 import hsgeneral as hs
from molspin_b200 import systems as S
from oracle import pyoracle as orc
from tests import helpers as h

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def _dense(system, F, times, precision, renorm=1, noise=None, propagator="dense", krylov=16):
    with hs.HSPropagatorB200(0) as p:
        p.set_hamiltonian(*system.hamiltonian_csr())
        p.set_reaction(kappa=system.kappa())
        p.set_electron_pair(*system.electron_strides())
        p.set_observables([(op, rate) for _, op, rate in system.observables()])
        p.set_option(L.OPT_DENSE_RENORMALIZE, renorm)
        if noise is not None:
            p.set_noise(*noise)
        p.set_factors(F)
        p.propagate(times, krylov, precision, propagator=propagator)
        per, ens = p.yields()
        return per, ens, p.values(), p.get_factors()


# (precision, per-trajectory tolerance, ensemble tolerance) after 300 steps at D=64
SMALL_TOL = [("bf16x3", 2e-4, 5e-5), ("bf16x6", 1e-5, 5e-6),  # measured 5.7e-5 / 2.4e-5 and 1.6e-6 / 6.5e-7
             ("int8x4", 1e-7, 1e-7)]


@pytest.mark.parametrize("precision,tol_traj,tol_ens", SMALL_TOL)
def test_dense_against_expm_oracle(precision, tol_traj, tol_ens):
    w = S.plain_small()
    M, steps = 96, 300
    times = S.time_grid(steps * w.dt, w.dt)
    F = w.system.trace_samples(M, w.seed)
    per, ens, values, _ = _dense(w.system, F, times, precision)
    ref = orc.hs_stochastic(w.system.hamiltonian_csr(), F, times, h.oracle_observables(w.system),
                            kappa=w.system.kappa(), method=1, nthreads=8)
    print(f"{precision}: traj {_rel(per, ref['traj_yield']):.3e} ens {_rel(ens, ref['yield']):.3e}")
    assert _rel(per, ref["traj_yield"]) < tol_traj
    assert _rel(ens, ref["yield"]) < tol_ens
    assert _rel(values, ref["values"]) < tol_traj


@pytest.mark.parametrize("precision,tol_traj,tol_ens", [("bf16x6", 5e-5, 2e-5), ("int8x4", 1e-7, 1e-7)])
def test_dense_with_philox_st_noise(precision, tol_traj, tol_ens):
    # singlet-triplet dephasing flips drawn on the device, replayed on the CPU
    system = h.random_system([2, 3], [2, 2], seed=12, st_rate=0.08, hf_scale=3.0)
    M, times = 70, S.time_grid(120.0, 1.0)
    F = system.trace_samples(M, 3.0)
    seed = 0xC0FFEE
    per, ens, _, _ = _dense(system, F, times, precision, noise=(system.st_rate, L.NOISE_PHILOX, seed))
    bits = hs.philox_flip_bits(seed, system.st_rate, times, M)
    ref = orc.hs_stochastic(system.hamiltonian_csr(), F, times, h.oracle_observables(system), kappa=system.kappa(),
                            method=1, U_csr=orc.st_unitary(system.mult, *system.electrons),
                            event_rate=0.5 * system.st_rate, noise_mode=1, flip_bits=bits, nthreads=8)
    assert bits.any()
    assert _rel(per, ref["traj_yield"]) < tol_traj
    assert _rel(ens, ref["yield"]) < tol_ens


def test_dense_norm_drift_and_renormalisation():
    # Haberkorn survival with K = k/2 I: |psi(t)|^2 = |psi(0)|^2 exp(-k t) exactly
    w = S.dense_tc(M=128, steps=200)
    times = S.time_grid(200 * w.dt, w.dt)
    F = w.system.trace_samples(128, w.seed)
    exact = np.sum(np.abs(F) ** 2, axis=0) * np.exp(-2.0 * w.system.kappa() * times[-1])
    for precision, max_drift in (("bf16x3", 2e-5), ("bf16x6", 2e-5), ("int8x4", 1e-9)):
        _, _, _, raw = _dense(w.system, F, times, precision, renorm=0)
        drift = np.max(np.abs(np.sum(np.abs(raw) ** 2, axis=0) / exact - 1.0)) / 200
        assert drift < max_drift, (precision, drift)  # per step; BF16 forms measured near 8e-6 at D=1024
        _, _, _, fixed = _dense(w.system, F, times, precision, renorm=1)
        assert np.max(np.abs(np.sum(np.abs(fixed) ** 2, axis=0) / exact - 1.0)) < 1e-6


# (precision, per-trajectory / values tolerance, ensemble tolerance) after 200 steps at D=1024
D1024_TOL = [("bf16x3", 1e-4, 5e-5), ("bf16x6", 2e-5, 1e-5),  # measured 2.8e-5 / 2.4e-5 and 4.0e-6 / 2.9e-6
             ("int8x4", 1e-7, 1e-7)]


@pytest.mark.parametrize("precision,tol_traj,tol_ens", D1024_TOL)
def test_dense_d1024_against_complex128_krylov(precision, tol_traj, tol_ens):
    # the dense form at the tensor-core workload's dimension against the FP64
    # Krylov form (pinned to the oracle at 1e-10) on the same trajectories
    w = S.dense_tc(M=256, steps=200)
    times = S.time_grid(200 * w.dt, w.dt)
    F = w.system.trace_samples(256, w.seed)
    per128, ens128, val128, _ = _dense(w.system, F, times, "c128", propagator="krylov", krylov=w.krylov)
    per, ens, values, _ = _dense(w.system, F, times, precision)
    print(f"{precision}: traj {_rel(per, per128):.3e} ens {_rel(ens, ens128):.3e} values {_rel(values, val128):.3e}")
    assert _rel(per, per128) < tol_traj
    assert _rel(ens, ens128) < tol_ens
    assert _rel(values, val128) < tol_traj


def test_dense_chunked_run_matches_one_run():
    # a run split into chunks (step_offset + accumulate) continues the noise
    # stream, the trapezoid and the per-time-point values of one long run
    system = h.random_system([2, 3], [2, 2], seed=12, st_rate=0.08, hf_scale=3.0)
    M, times = 70, S.time_grid(60.0, 1.0)
    F = system.trace_samples(M, 3.0)
    noise = (system.st_rate, L.NOISE_PHILOX, 4242)
    with hs.HSPropagatorB200(0) as p:
        p.set_hamiltonian(*system.hamiltonian_csr())
        p.set_reaction(kappa=system.kappa())
        p.set_electron_pair(*system.electron_strides())
        p.set_observables([(op, rate) for _, op, rate in system.observables()])
        p.set_noise(*noise)
        p.set_factors(F)
        p.propagate(times, 16, "bf16x6", propagator="dense")
        per1, ens1 = p.yields()
        val1 = p.values()
        p.set_factors(F)
        vals, start = [], 0
        for k, stop in enumerate([17, 33, 60]):
            p.propagate(times[start:stop + 1], 16, "bf16x6", step_offset=start, accumulate=k > 0, propagator="dense")
            vals.append(p.values() if k == 0 else p.values()[1:])
            start = stop
        per2, ens2 = p.yields()
        val2 = np.concatenate(vals)
    assert _rel(per2, per1) < 1e-6
    assert _rel(ens2, ens1) < 1e-6
    assert _rel(val2, val1) < 1e-6


def test_dense_error_paths():
    w = S.plain_small()
    F = w.system.trace_samples(8, w.seed)
    with hs.HSPropagatorB200(0) as p:
        p.set_hamiltonian(*w.system.hamiltonian_csr())
        p.set_reaction(kappa=w.system.kappa())
        p.set_electron_pair(*w.system.electron_strides())
        p.set_observables([(op, rate) for _, op, rate in w.system.observables()])
        p.set_factors(F)
        with pytest.raises(hs.MsgpuError) as e:
            p.propagate(S.time_grid(4.0, 1.0), 8, "c128", propagator="dense")
        assert e.value.code == L.MSGPU_ERR_INVALID
        with pytest.raises(hs.MsgpuError) as e:
            p.propagate(np.array([0.0, 1.0, 2.5, 3.0]), 8, "bf16x3", propagator="dense")
        assert e.value.code == L.MSGPU_ERR_INVALID
        # the context stays usable after a rejected call
        p.propagate(S.time_grid(4.0, 1.0), 8, "bf16x3", propagator="dense")
    big = h.random_system([2] * 6, [2] * 5, seed=2, aniso=False)  # D = 8192
    with hs.HSPropagatorB200(0) as p:
        p.set_hamiltonian(*big.hamiltonian_csr())
        p.set_reaction(kappa=big.kappa())
        p.set_electron_pair(*big.electron_strides())
        p.set_observables([(op, rate) for _, op, rate in big.observables()])
        p.set_factors(big.trace_samples(2, 1.0))
        with pytest.raises(hs.MsgpuError) as e:
            p.propagate(S.time_grid(2.0, 1.0), 8, "bf16x3", propagator="dense")
        assert e.value.code == L.MSGPU_ERR_INVALID
