"""Batching form (msgpu_batch_*): several systems of uneven dimension in one
persistent launch, against the CPU oracle and against itself in other mixes.

Tolerance: complex64 vectors with FP64 reductions -> per-trajectory yields
within 1e-6 of the largest per-trajectory yield of the complex128 oracle.
"""
import numpy as np
import pytest

from molspin_b200 import _lib as L
from molspin_b200 import batching as B
from molspin_b200 import hsgeneral as hs
from molspin_b200 import systems as S
from oracle import pyoracle as orc
from tests import helpers as h

pytestmark = pytest.mark.gpu


def _systems():
    a = h.random_system([2, 2], [], seed=51, st_rate=0.05, hf_scale=2.0, aniso=False)           # D = 16
    b = h.random_system([2, 3], [2], seed=52, st_rate=0.02, hf_scale=2.0, aniso=False)          # D = 48
    c = h.random_system([2, 2, 2, 2], [2, 2, 2], seed=53, st_rate=0.03, hf_scale=2.0, aniso=False)  # D = 512
    return [(a, 40, 11), (b, 70, 12), (c, 33, 13)]


def _run(entries, times, krylov, chunks=None, tune=False):
    with B.BatchB200(0) as bt:
        idx = [bt.add(s, s.trace_samples(M, float(seed)), seed) for s, M, seed in entries]
        if tune:
            bt.tune(times[:4], krylov)
        if chunks is None:
            bt.run(times, krylov)
        else:
            start = 0
            for k, stop in enumerate(chunks):
                bt.run(times[start:stop + 1], krylov, step_offset=start, accumulate=k > 0)
                start = stop
        stats = bt.stats()
        stats["systems"] = [bt.system_info(i) for i in idx]
        return [bt.yields(i) for i in idx], stats


def test_batch_matches_oracle():
    entries = _systems()
    times = S.time_grid(30.0, 1.0)
    m = 12
    out, stats = _run(entries, times, m, tune=True)
    assert stats["team_threshold"] > 0
    for (s, M, seed), (per, ens) in zip(entries, out):
        F = s.trace_samples(M, float(seed))
        bits = hs.philox_flip_bits(seed, s.st_rate, times, M)
        ref = orc.hs_stochastic(s.hamiltonian_csr(), F, times, h.oracle_observables(s), kappa=s.kappa(), krylov=m,
                                U_csr=orc.st_unitary(s.mult, 0, 1), event_rate=0.5 * s.st_rate, noise_mode=1,
                                flip_bits=bits, nthreads=8)
        scale = np.max(np.abs(ref["traj_yield"]))
        assert np.max(np.abs(per - ref["traj_yield"])) <= 1e-6 * scale, s.dim


def test_batch_result_independent_of_companions_and_chunks():
    entries = _systems()
    times = S.time_grid(20.0, 1.0)
    alone, _ = _run(entries[2:], times, 10)
    mixed, _ = _run(entries, times, 10)
    np.testing.assert_array_equal(alone[0][0], mixed[2][0])
    chunked, _ = _run(entries, times, 10, chunks=[7, 20])
    for x, y in zip(mixed, chunked):
        np.testing.assert_array_equal(x[0], y[0])


def test_cleared_batch_reuses_its_buffers_and_matches_fresh_batches():
    # a batch cleared between groups of systems (msgpu_batch_clear keeps the
    # persistent route's device buffers) gives each group the result of a
    # fresh batch, bit for bit, including a group smaller than the first
    entries = _systems()
    times = S.time_grid(20.0, 1.0)
    fresh_all, _ = _run(entries, times, 10)
    fresh_one, _ = _run(entries[1:2], times, 10)
    with B.BatchB200(0) as bt:
        for group, ref in ((entries, fresh_all), (entries[1:2], fresh_one), (entries, fresh_all)):
            bt.clear()
            idx = [bt.add(s, s.trace_samples(M, float(seed)), seed) for s, M, seed in group]
            bt.run(times, 10)
            for i, (per, ens) in zip(idx, ref):
                got = bt.yields(i)
                np.testing.assert_array_equal(got[0], per)
                np.testing.assert_array_equal(got[1], ens)


def test_batch_streams_large_systems_through_the_single_system_path():
    # D = 2048 reaches the streamed threshold: it runs on its own context
    # beside the persistent launch, and equals the single-system complex64 run
    big = h.random_system([2] * 5, [2] * 4, seed=54, st_rate=0.03, hf_scale=2.0, aniso=False)
    assert big.dim == 2048
    entries = [_systems()[0], (big, 45, 14)]
    times = S.time_grid(12.0, 1.0)
    m = 10
    out, stats = _run(entries, times, m, tune=True)
    # the small system runs in the persistent launch; the large one on its own
    # context, whose tuner picked an SpMM variant, tile and trajectory grouping
    small_info, big_info = stats["systems"]
    assert not small_info["streamed"] and small_info["spmm_variant"] == -1
    assert big_info["streamed"] and big_info["spmm_variant"] >= 0 and big_info["spmm_tile"] > 0
    assert big_info["traj_groups"] >= 1
    F = big.trace_samples(45, 14.0)
    with hs.HSPropagatorB200(0) as p:
        p.set_hamiltonian(*big.hamiltonian_csr())
        p.set_reaction(kappa=big.kappa())
        p.set_electron_pair(*big.electron_strides())
        p.set_observables([(op, rate) for _, op, rate in big.observables()])
        p.set_noise(big.st_rate, L.NOISE_PHILOX, 14)
        p.set_factors(F)
        p.propagate(times, m, "c64")
        per, ens = p.yields()
    np.testing.assert_array_equal(out[1][0], per)
    np.testing.assert_array_equal(out[1][1], ens)
    bits = hs.philox_flip_bits(14, big.st_rate, times, 45)
    ref = orc.hs_stochastic(big.hamiltonian_csr(), F, times, h.oracle_observables(big), kappa=big.kappa(), krylov=m,
                            U_csr=orc.st_unitary(big.mult, 0, 1), event_rate=0.5 * big.st_rate, noise_mode=1,
                            flip_bits=bits, nthreads=8)
    assert np.max(np.abs(out[1][0] - ref["traj_yield"])) <= 1e-6 * np.max(np.abs(ref["traj_yield"]))
