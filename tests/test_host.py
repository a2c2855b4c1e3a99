"""Host-side helpers of libmsgpu (no GPU): Hamiltonian assembly, trace
sampling, flip streams and the time grid against independent restatements."""
import math

import numpy as np

from molspin_b200 import hsgeneral as hs
from molspin_b200 import systems as S
from oracle import density as den
from oracle import pyoracle as orc
from tests import helpers as h


def _dense_from_csr(rowptr, col, val, D):
    A = np.zeros((D, D), complex)
    for r in range(D):
        A[r, col[rowptr[r]:rowptr[r + 1]]] += val[rowptr[r]:rowptr[r + 1]]
    return A


def test_hamiltonian_matches_dense_kronecker():
    cases = [
        h.random_system([2, 2], [2], seed=1, aniso=False),
        h.random_system([2, 3, 2], [2, 3], seed=2, aniso=True),
        S.plain_small().system,
    ]
    for system in cases:
        r, c, v = system.hamiltonian_csr()
        H = _dense_from_csr(r, c, v, system.dim)
        ref = den.dense_hamiltonian(system)
        assert np.linalg.norm(H - ref) <= 1e-12 * np.linalg.norm(ref)
        assert np.linalg.norm(H - H.conj().T) <= 1e-14 * np.linalg.norm(H)
        assert np.all(np.diff(r) >= 0) and all(np.all(np.diff(c[r[i]:r[i + 1]]) > 0) for i in range(system.dim))


def test_hamiltonian_with_permuted_spin_order():
    # electrons not leading; reversed bilinear roles
    s = S.SpinSystem(mult=[2, 2, 3, 2], names=["N1", "E1", "N2", "E2"], electrons=(1, 3))
    rng = np.random.default_rng(3)
    s.linear = [(1, rng.normal(size=3)), (3, rng.normal(size=3))]
    s.bilinear = [(1, 0, rng.normal(size=(3, 3))), (2, 3, rng.normal(size=(3, 3)))]
    r, c, v = s.hamiltonian_csr()
    H = _dense_from_csr(r, c, v, s.dim)
    ref = den.dense_hamiltonian(s)
    assert np.linalg.norm(H - ref) <= 1e-12 * np.linalg.norm(ref)


def test_config_shapes_and_nnz():
    w = S.precision_large(M=8, steps=1)
    assert w.system.dim == 16384
    r, c, v = w.system.hamiltonian_csr()
    assert len(r) == 16385
    # anisotropic couplings + tilted field: 1 + 2 + 2*12 = 27 entries per row
    assert np.max(np.diff(r)) == 27
    assert S.plain_small().system.dim == 64
    assert S.dense_tc(M=8, steps=1).system.dim == 1024


def test_trace_samples_match_oracle_bitwise():
    w = S.plain_small()
    F = w.system.trace_samples(16, 1.0)
    G = orc.trace_samples(1.0, S.SINGLET, 16, 16)
    np.testing.assert_array_equal(F, G)
    assert np.allclose(np.linalg.norm(F, axis=0), 1 / math.sqrt(16), atol=1e-15)


def test_reference_flip_bits_match_oracle_bitwise():
    times = orc.time_grid(3.0, 0.25)
    for seed_mode in (0, 1):
        a = hs.reference_flip_bits(431.0, 0.7, times, 37, orientation=2, seed_mode=seed_mode)
        b = orc.st_flip_bits(431.0, seed_mode, 2, 0.35, times, 37)
        np.testing.assert_array_equal(a, b)


def test_philox_flip_rate():
    times = np.arange(201, dtype=float)
    M = 512
    st = 0.05
    bits = hs.philox_flip_bits(1234, st, times, M)
    n = np.unpackbits(bits, bitorder="little")[: 200 * 2 * M].sum()
    p = -0.5 * math.expm1(-2 * 0.5 * st * 0.5)
    N = 200 * 2 * M
    assert abs(n / N - p) < 6 * math.sqrt(p * (1 - p) / N)
    # counter-based: a trajectory's bits do not depend on the block it is in
    sub = hs.philox_flip_bits(1234, st, times, 64, traj_offset=100)
    full = np.unpackbits(bits, bitorder="little")[: 200 * 2 * M].reshape(400, M)
    part = np.unpackbits(sub, bitorder="little")[: 200 * 2 * 64].reshape(400, 64)
    np.testing.assert_array_equal(full[:, 100:164], part)


def test_time_grid_matches_oracle():
    for total, dt in [(5000.0, 1.0), (2.0, 0.025), (0.1, 0.03), (3.0, 0.7)]:
        np.testing.assert_array_equal(S.time_grid(total, dt), orc.time_grid(total, dt))


def test_plan_validation():
    import pytest
    with pytest.raises(ValueError):
        hs.HSExecutionPlan(timestep=0.0).validate()
    with pytest.raises(ValueError):
        hs.HSExecutionPlan(gpuprecision="fp16").validate()
    p = hs.HSExecutionPlan(krylovsize=0)
    p.validate()
    assert p.krylovsize == 16
    assert abs(hs.yield_correction(0.5, 0.02) - orc.yield_correction(0.5, 0.02)) < 1e-15


def test_field_terms_reproduce_the_hamiltonian():
    # H_0 + Bx Zx + By Zy + Bz Zz on the union pattern equals H(B) built directly
    rng = np.random.default_rng(21)
    ta = [S._aniso_tensor(rng, 1.5) for _ in range(2)]
    tb = [S._aniso_tensor(rng, 1.5)]
    B = np.array([12e-6, -30e-6, 41e-6])
    direct = S.radical_pair([2, 2], [2], ta, tb, B, sink_rate=1e-3)
    r, c, v = S.field_terms(direct)
    coef = np.array([1.0, *B])
    D = direct.dim
    combined = np.zeros((D, D), dtype=np.complex128)
    for k in range(4):
        for row in range(D):
            for idx in range(r[row], r[row + 1]):
                combined[row, c[idx]] += coef[k] * v[k, idx]
    rd, cd, vd = direct.hamiltonian_csr()
    ref = np.zeros((D, D), dtype=np.complex128)
    for row in range(D):
        for idx in range(rd[row], rd[row + 1]):
            ref[row, cd[idx]] += vd[idx]
    assert np.max(np.abs(combined - ref)) < 1e-12 * np.max(np.abs(ref))
    assert v.shape == (4, r[-1])


def test_multi_term_flip_stream_matches_oracle_and_law():
    # several dephasing Operators on one pair: superposed Poisson counts with
    # channel marks, parity bits; bitwise equal to the oracle, reduces to the
    # Bernoulli stream for one term, and flips with p = (1 - exp(-2 L h)) / 2
    times = S.time_grid(40.0, 1.0)
    M = 300
    for rates, seed, orient in (([0.3, 0.5], 7.0, 0), ([0.1, 0.2, 0.05], 2.0, 5)):
        host = hs.reference_flip_bits_multi(seed, rates, times, M, orient)
        ref = orc.st_flip_bits_multi(seed, 0, orient, [0.5 * r for r in rates], times, M)
        np.testing.assert_array_equal(host, ref)
        total = 0.5 * sum(rates)
        p = -0.5 * np.expm1(-2.0 * total * 0.5)
        frac = np.unpackbits(host, bitorder="little")[: (len(times) - 1) * 2 * M].mean()
        assert abs(frac - p) < 6.0 * math.sqrt(p * (1 - p) / ((len(times) - 1) * 2 * M))
    one = hs.reference_flip_bits_multi(3.0, [0.4], times, M, 2)
    np.testing.assert_array_equal(one, hs.reference_flip_bits(3.0, 0.4, times, M, 2))
