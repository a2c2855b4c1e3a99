"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

Tolerances (written per test): per-trajectory yields of the complex128 form
within 1e-10 relative of the oracle; exact-trace ensembles within 1e-10 of
the density oracle; stochastic ensembles within the reference's 6 sigma bound
6/(2 sqrt(M)); Haberkorn survival within 2e-6 (reference bound).
"""
import math

import numpy as np
import pytest

from molspin_b200 import _lib as L
from molspin_b200 import hsgeneral as hs
from molspin_b200 import systems as S
from oracle import density as den
from oracle import pyoracle as orc
from tests import helpers as h

pytestmark = pytest.mark.gpu


FORMS = ["streamed", "resident"]


def _gpu(system, factors, times, krylov, precision="c128", noise=None, K_csr=None, kappa=None,
         obs=None, chunks=None, form="auto", propagator="krylov"):
    with hs.HSPropagatorB200(0) as p:
        p.set_form(form)
        p.set_hamiltonian(*system.hamiltonian_csr())
        if K_csr is not None:
            p.set_reaction(csr=K_csr)
        else:
            p.set_reaction(kappa=system.kappa() if kappa is None else kappa)
        p.set_electron_pair(*system.electron_strides())
        obs = obs if obs is not None else [(op, rate) for _, op, rate in system.observables()]
        p.set_observables(obs)
        if noise is not None:
            p.set_noise(*noise)
        p.set_factors(factors)
        if chunks is None:
            p.propagate(times, krylov, precision, propagator=propagator)
            values = p.values()
        else:
            values = []
            start = 0
            for k, stop in enumerate(chunks):
                p.propagate(times[start:stop + 1], krylov, precision, step_offset=start, accumulate=k > 0)
                values.append(p.values() if k == 0 else p.values()[1:])
                start = stop
            values = np.concatenate(values)
        per, ens = p.yields()
        return per, ens, values, p.get_factors()


def _oracle(system, factors, times, krylov, U=False, **kw):
    obs = h.oracle_observables(system)
    if U:
        kw["U_csr"] = orc.st_unitary(system.mult, *system.electrons)
        kw["event_rate"] = 0.5 * system.st_rate
    return orc.hs_stochastic(system.hamiltonian_csr(), factors, times, obs, krylov=krylov, nthreads=8, **kw)


def _rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


@pytest.mark.parametrize("form", FORMS)
def test_plain_per_trajectory_parity_config1_shape(form):
    w = S.plain_small()
    M, steps = 64, 200
    times = S.time_grid(steps * w.dt, w.dt)
    F = w.system.trace_samples(M, w.seed)
    per, ens, values, Fg = _gpu(w.system, F, times, w.krylov, form=form)
    ref = _oracle(w.system, F, times, w.krylov, kappa=w.system.kappa())
    assert _rel(per, ref["traj_yield"]) < 1e-10
    assert _rel(ens, ref["yield"]) < 1e-10
    assert _rel(values, ref["values"]) < 1e-10
    assert np.max(np.abs(Fg - ref["factors"])) < 1e-10 * np.max(np.abs(ref["factors"]))


@pytest.mark.parametrize("form", FORMS)
def test_plain_parity_reference_noise_stream(form):
    system = h.random_system([2, 2, 2], [2], seed=11, st_rate=0.05, sink=2e-3, hf_scale=3.0)
    M, times = 100, S.time_grid(60.0, 0.5)
    F = system.trace_samples(M, 7.0)
    bits = hs.reference_flip_bits(7.0, system.st_rate, times, M, orientation=0)
    assert np.unpackbits(bits).sum() > 50
    per, ens, _, _ = _gpu(system, F, times, 12, noise=(system.st_rate, L.NOISE_REPLAY, 0, bits, len(times) - 1, M),
                          form=form)
    ref = _oracle(system, F, times, 12, U=True, kappa=system.kappa(), noise_mode=0, seed=7.0, seed_mode=0)
    assert _rel(per, ref["traj_yield"]) < 1e-10
    assert _rel(ens, ref["yield"]) < 1e-10


@pytest.mark.parametrize("form", FORMS)
def test_plain_parity_philox_replayed_on_cpu(form):
    system = h.random_system([2, 3], [2, 2], seed=12, st_rate=0.08, hf_scale=3.0)
    M, times = 70, S.time_grid(40.0, 1.0)
    F = system.trace_samples(M, 3.0)
    seed = 0xDEADBEEF1234
    per, ens, _, _ = _gpu(system, F, times, 16, noise=(system.st_rate, L.NOISE_PHILOX, seed), form=form)
    bits = hs.philox_flip_bits(seed, system.st_rate, times, M)
    ref = _oracle(system, F, times, 16, U=True, kappa=system.kappa(), noise_mode=1, flip_bits=bits)
    assert _rel(per, ref["traj_yield"]) < 1e-10


@pytest.mark.parametrize("form", FORMS)
def test_plain_parity_general_K_and_interleaved_electrons(form):
    # electrons at positions 1 and 3 (neither leading), unequal sinks -> CSR K
    s = S.SpinSystem(mult=[2, 2, 3, 2, 2], names=["N1", "E1", "N2", "E2", "N3"], electrons=(1, 3))
    rng = np.random.default_rng(4)
    for e in (1, 3):
        s.linear.append((e, S.COMMON_PREFACTOR * 2.0023 * 1e-4 * rng.normal(size=3)))
    for e, n in ((1, 0), (1, 2), (3, 4)):
        s.bilinear.append((e, n, S.COMMON_PREFACTOR * 2.0023e-3 * S._aniso_tensor(rng, 2.0)))
    s.sinks = {"S": 3e-3, "T0": 1e-3, "Tp": 1e-3, "Tm": 1e-3}
    s.st_rate = 0.0
    K = sum(0.5 * rate * den.pair_operator(S.pair_projector(S.PAIR_STATES[n]), s) for n, rate in s.sinks.items())
    Kc = den.to_csr(K, 1e-18)
    M = 45
    F = rng.normal(size=(s.dim, M)) + 1j * rng.normal(size=(s.dim, M))
    F /= np.linalg.norm(F, axis=0) * math.sqrt(M)
    times = S.time_grid(30.0, 1.0)
    obs = [(op, rate) for _, op, rate in s.observables()]
    per, ens, _, _ = _gpu(s, F, times, 10, K_csr=Kc, obs=obs, form=form)
    ref = orc.hs_stochastic(s.hamiltonian_csr(), F, times, h.oracle_observables(s), K_csr=Kc, krylov=10)
    assert _rel(per, ref["traj_yield"]) < 1e-10


@pytest.mark.parametrize("form", FORMS)
def test_exact_trace_against_density_oracle(form):
    system = h.random_system([2, 2], [2], seed=21, hf_scale=2.0)
    times = S.time_grid(80.0, 1.0)
    F = den.orthonormal_nuclear_samples(system, S.SINGLET)
    _, ens, values, _ = _gpu(system, F, times, 16, form=form)
    H = den.dense_hamiltonian(system)
    K = system.kappa() * np.eye(system.dim)
    ops = [(den.pair_operator(op, system), rate) for _, op, rate in system.observables()]
    dv, dy = den.propagate_density(H, K, den.singlet_density(system), times, ops)
    assert _rel(ens, dy) < 1e-10
    assert _rel(values, dv) < 1e-10


@pytest.mark.parametrize("propagator", ["krylov", "taylor"])
def test_stochastic_st_against_lindblad_and_survival(propagator):
    # The reference's Tests/StochasticRelaxation/st_dephasing.msd on the GPU: 8192 samples with
    # seed 431, dt 0.025 over 2 ns, its stochastic task's propagationmethod=autoexpm with
    # precision=double (the Taylor propagator) and the Krylov step (m=8), with the reference's
    # own flip stream replayed.  The population difference from the direct task must equal the
    # value the reference recorded for this example, and survival must be at its 1e-12 level.
    system = h.st_fixture()
    times = S.time_grid(2.0, 0.025)
    M = 8192
    F = system.trace_samples(M, 431.0)
    pops = [(S.pair_projector(S.PAIR_STATES[n]), 1.0) for n in ("S", "T0", "Tp", "Tm")]
    bits = hs.reference_flip_bits(431.0, 0.7, times, M)
    _, _, values, _ = _gpu(system, F, times, 8, noise=(0.7, L.NOISE_REPLAY, 0, bits, len(times) - 1, M), obs=pops,
                           propagator=propagator)
    assert values.shape == (81, 4)
    surv = np.max(np.abs(values.sum(axis=1) - np.exp(-0.2 * times)))
    assert surv < 1e-11, surv  # the reference recorded 8.129053e-13 (check_output.py bound: 2e-6)
    # the reference's recorded population error of this example against its direct task
    # (density-matrix RK4), STOCHASTIC_RELAXATION.md:250-251: 0.0012766377
    err = den.data_file_difference(values, h.st_dephasing_direct(system, times))
    assert abs(err - h.ST_DEPHASING_POPULATION_ERROR) < h.ST_DEPHASING_PIN_TOL, err
    assert err < h.six_sigma(M)


@pytest.mark.parametrize("form", FORMS)
def test_chunked_run_is_bitwise_identical(form):
    system = h.random_system([2, 2, 2], [2, 2], seed=31, st_rate=0.05, hf_scale=2.0)
    M, times = 64, S.time_grid(40.0, 1.0)
    F = system.trace_samples(M, 5.0)
    noise = (system.st_rate, L.NOISE_PHILOX, 99)
    a = _gpu(system, F, times, 12, noise=noise, form=form)
    b = _gpu(system, F, times, 12, noise=noise, chunks=[13, 27, 40], form=form)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[2], b[2])


def test_resident_precision_form_against_plain():
    # complex64 Lanczos in shared memory vs the complex128 Arnoldi path
    system = h.random_system([2, 2, 2, 2], [2, 2, 2], seed=41, st_rate=0.05, hf_scale=2.0)
    M, times = 96, S.time_grid(100.0, 1.0)
    F = system.trace_samples(M, 9.0)
    noise = (system.st_rate, L.NOISE_PHILOX, 7)
    per64, ens64, val64, _ = _gpu(system, F, times, 16, precision="c64", noise=noise, form="resident")
    per128, ens128, val128, _ = _gpu(system, F, times, 16, precision="c128", noise=noise, form="resident")
    assert abs(ens64[0] - ens128[0]) <= 1e-6 * abs(ens128[0])
    assert np.max(np.abs(val64 - val128)) <= 1e-6 * np.max(np.abs(val128))


def test_precision_form_against_plain():
    w = S.precision_large(M=64, steps=40)
    F = w.system.trace_samples(64, 1.0)
    times = S.time_grid(40 * w.dt, w.dt)
    per64, ens64, val64, _ = _gpu(w.system, F, times, w.krylov, precision="c64")
    per128, ens128, val128, _ = _gpu(w.system, F, times, w.krylov, precision="c128")
    # singlet yield (observable 0): ensemble within 1e-6 relative of the complex128 path
    assert abs(ens64[0] - ens128[0]) <= 1e-6 * abs(ens128[0])
    assert np.max(np.abs(val64 - val128)) <= 1e-6 * np.max(np.abs(val128))


def test_full_size_survival_property():
    # size-independent law at the benchmark size D=16384: with K = k/2 I the
    # population summed over S, T0, T+, T- decays exactly as exp(-k t)
    w = S.precision_large(M=64, steps=6)
    F = w.system.trace_samples(64, 1.0)
    times = S.time_grid(6 * w.dt, w.dt)
    k = 1e-3
    pops = [(S.pair_projector(S.PAIR_STATES[n]), 1.0) for n in ("S", "T0", "Tp", "Tm")]
    for prec, tol in (("c128", 1e-12), ("c64", 2e-6)):
        _, _, values, _ = _gpu(w.system, F, times, w.krylov, precision=prec, obs=pops)
        assert np.max(np.abs(values.sum(axis=1) - np.exp(-k * times))) < tol


def test_error_paths():
    system = h.random_system([2, 2], [2], seed=3)
    r, c, v = system.hamiltonian_csr()
    with hs.HSPropagatorB200(0) as p:
        bad = v.copy()
        bad[0] = np.nan
        with pytest.raises(hs.MsgpuError) as e:
            p.set_hamiltonian(r, c, bad)
        assert e.value.code == L.MSGPU_ERR_NONFINITE
        with pytest.raises(hs.MsgpuError) as e:
            p.propagate(S.time_grid(2.0, 1.0), 8)
        assert e.value.code == L.MSGPU_ERR_STATE
        p.set_hamiltonian(r, c, v)
        with pytest.raises(hs.MsgpuError) as e:
            p.set_electron_pair(4, 4)
        assert e.value.code == L.MSGPU_ERR_INVALID
    with hs.HSPropagatorB200(0, hbm_budget=4096) as p:
        with pytest.raises(hs.MsgpuError) as e:
            p.set_hamiltonian(r, c, v)
            p.set_factors(system.trace_samples(64, 1.0))
        assert e.value.code == L.MSGPU_ERR_BUDGET


def test_multi_term_dephasing_stream_replayed():
    # two dephasing Operators on the pair: the reference's superposed-Poisson
    # stream as parity bits, replayed on the device against the oracle
    system = h.random_system([2, 3], [2, 2], seed=12, st_rate=0.0, hf_scale=3.0)
    rates = [0.05, 0.08]
    system.st_rate = sum(rates)
    M, times = 40, S.time_grid(40.0, 1.0)
    F = system.trace_samples(M, 3.0)
    bits = hs.reference_flip_bits_multi(9.0, rates, times, M, 1)
    assert bits.any()
    per, ens, _, _ = _gpu(system, F, times, 16, noise=(system.st_rate, L.NOISE_REPLAY, 0, bits, len(times) - 1, M))
    ref = _oracle(system, F, times, 16, U=True, kappa=system.kappa(), noise_mode=1, flip_bits=bits)
    assert _rel(per, ref["traj_yield"]) < 1e-10
    # the complex64 form (streamed Lanczos) replays the same parity bits
    per64, _, _, _ = _gpu(system, F, times, 16, precision="c64", form="streamed",
                          noise=(system.st_rate, L.NOISE_REPLAY, 0, bits, len(times) - 1, M))
    assert _rel(per64, ref["traj_yield"]) < 1e-6


def test_multi_term_dephasing_philox_is_the_summed_rate():
    # Every channel applies P_S - P_T, so only the parity of the superposed
    # Poisson count acts; its odd probability is the one-channel formula at
    # the summed rate.  The device's Philox stream at the summed rate against
    # the exact density-matrix yield (the Lindblad sum of the channels), both
    # precisions, within 5 standard errors of the trajectory mean.
    system = h.random_system([2, 2], [2], seed=14, st_rate=0.0, hf_scale=2.0)  # D = 32
    rates = [0.2, 0.3]
    system.st_rate = sum(rates)
    M, times = 4096, S.time_grid(20.0, 0.5)
    F = system.trace_samples(M, 5.0)
    H = den.dense_hamiltonian(system)
    K = system.kappa() * np.eye(system.dim)
    ops = [(den.pair_operator(op, system), rate) for _, op, rate in system.observables()]
    _, ref = den.propagate_density(H, K, den.singlet_density(system), times, ops, U=den.st_unitary(system),
                                   st_rate=system.st_rate)
    for precision in ("c128", "c64"):
        per, ens, _, _ = _gpu(system, F, times, 16, precision=precision, form="streamed",
                              noise=(system.st_rate, L.NOISE_PHILOX, 41))
        se = np.std(per, axis=0) * np.sqrt(M)
        assert np.all(np.abs(ens - ref) < 5 * se + 1e-12), (precision, ens, ref, se)


@pytest.mark.parametrize("variant", [4, 5, 6, 7])
def test_shared_memory_spmm_variants(variant):
    # the SpMM variants that stage the tile's own quartets in shared memory,
    # forced: complex64 against complex128 within the precision form's 1e-6
    # and against the register-gather variant to FP32 rounding
    system = h.random_system([2] * 5, [2] * 3, seed=71, aniso=True, st_rate=0.05)  # D = 1024
    M, times = 128, S.time_grid(30.0, 1.0)
    F = system.trace_samples(M, 2.0)
    noise = (system.st_rate, L.NOISE_PHILOX, 5)

    def run(precision, v):
        with hs.HSPropagatorB200(0) as p:
            p.set_form("streamed")
            if v is not None:
                p.set_option(L.OPT_SPMM_VARIANT, v)
            p.set_hamiltonian(*system.hamiltonian_csr())
            p.set_reaction(kappa=system.kappa())
            p.set_electron_pair(*system.electron_strides())
            p.set_observables([(op, rate) for _, op, rate in system.observables()])
            p.set_noise(*noise)
            p.set_factors(F)
            p.propagate(times, 16, precision)
            return p.yields()[0]

    cube = run("c64", variant)
    ref128 = run("c128", None)
    reg = run("c64", 3)
    assert _rel(cube, ref128) < 1e-6
    assert _rel(cube, reg) < 1e-6


def _unequal_sinks_system(n_a, n_b, seed):
    s = h.random_system(n_a, n_b, seed=seed, aniso=True, st_rate=0.05)
    s.sinks = {"S": 3e-3, "T0": 1e-3, "Tp": 0.5e-3, "Tm": 2e-3}
    K = sum(0.5 * rate * den.pair_operator(S.pair_projector(S.PAIR_STATES[n]), s) for n, rate in s.sinks.items())
    return s, den.to_csr(K, 1e-18)


def test_complex64_arnoldi_unequal_sinks_against_oracle():
    # unequal sinks make K = sum_c k_c/2 P_c a non-scalar operator on the pair:
    # the complex64 form runs Arnoldi (CGS2, FP64 dots, FP32 storage) and
    # matches the oracle's complex128 MGS Arnoldi within 1e-6 (a spin-1
    # nucleus, interleaved electrons)
    s = S.SpinSystem(mult=[2, 2, 3, 2, 2], names=["N1", "E1", "N2", "E2", "N3"], electrons=(1, 3))
    rng = np.random.default_rng(4)
    for e in (1, 3):
        s.linear.append((e, S.COMMON_PREFACTOR * 2.0023 * 1e-4 * rng.normal(size=3)))
    for e, n in ((1, 0), (1, 2), (3, 4)):
        s.bilinear.append((e, n, S.COMMON_PREFACTOR * 2.0023e-3 * S._aniso_tensor(rng, 2.0)))
    s.sinks = {"S": 3e-3, "T0": 1e-3, "Tp": 1e-3, "Tm": 1e-3}
    s.st_rate = 0.0
    K = sum(0.5 * rate * den.pair_operator(S.pair_projector(S.PAIR_STATES[n]), s) for n, rate in s.sinks.items())
    Kc = den.to_csr(K, 1e-18)
    M = 45
    F = rng.normal(size=(s.dim, M)) + 1j * rng.normal(size=(s.dim, M))
    F /= np.linalg.norm(F, axis=0) * math.sqrt(M)
    times = S.time_grid(30.0, 1.0)
    obs = [(op, rate) for _, op, rate in s.observables()]
    per, ens, vals, _ = _gpu(s, F, times, 10, precision="c64", K_csr=Kc, obs=obs, form="streamed")
    ref = orc.hs_stochastic(s.hamiltonian_csr(), F, times, h.oracle_observables(s), K_csr=Kc, krylov=10)
    assert _rel(per, ref["traj_yield"]) < 1e-6
    assert _rel(vals, ref["values"]) < 1e-6


def test_complex64_arnoldi_against_complex128_at_d1024():
    # D = 1024, unequal sinks, Philox ST noise, 256 trajectories over 60 steps:
    # complex64 Arnoldi against complex128 Arnoldi within the precision form's 1e-6
    s, Kc = _unequal_sinks_system([2] * 5, [2] * 3, 33)
    M, times = 256, S.time_grid(60.0, 1.0)
    F = s.trace_samples(M, 3.0)
    noise = (s.st_rate, L.NOISE_PHILOX, 19)
    per64, ens64, val64, _ = _gpu(s, F, times, 16, precision="c64", K_csr=Kc, noise=noise, form="streamed")
    per128, ens128, val128, _ = _gpu(s, F, times, 16, precision="c128", K_csr=Kc, noise=noise, form="streamed")
    assert _rel(per64, per128) < 1e-6
    assert np.max(np.abs(ens64 - ens128) / np.abs(ens128)) < 1e-6
    assert _rel(val64, val128) < 1e-6


def test_complex64_refuses_a_K_beyond_the_pair():
    # a K that couples nuclear states is not I x K4: complex64 refuses it, complex128 runs it
    s, Kc = _unequal_sinks_system([2, 2], [2], 35)
    r, c, v = Kc
    v = np.array(v, copy=True)
    v[0] *= 1.5  # the first quartet's block differs from the others
    F = s.trace_samples(64, 1.0)
    with pytest.raises(hs.MsgpuError) as e:
        _gpu(s, F, S.time_grid(3.0, 1.0), 8, precision="c64", K_csr=(r, c, v), form="streamed")
    assert e.value.code == L.MSGPU_ERR_INVALID
    _gpu(s, F, S.time_grid(3.0, 1.0), 8, precision="c128", K_csr=(r, c, v), form="streamed")
