"""The committed golden fixtures (tests/golden/*.npz, made by
tests/golden/make_golden.py) against the CPU oracle and the host helpers.

The oracle must reproduce its own committed outputs on the committed inputs
(relative 1e-12: the same algorithm, possibly another compiler), and the
product's host helpers must reproduce the committed inputs: H assembly
(SpinSpace_hamiltonians.cpp:438-777) within 1e-14 of the dense Kronecker
assembly, the trace samples (SpinSpace_states.cpp:452-486) and the
reference's flip stream (SpinSpace_relaxation.cpp:1201-1254) bit for bit.
"""
import os

import numpy as np
import pytest

from molspin_b200 import hsgeneral as hs
from molspin_b200 import systems as S
from oracle import density as den
from oracle import pyoracle as orc
from tests import helpers as h

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["plain_small", "st_noise", "exact_trace", "dense_branch"]


def load(name):
    with np.load(os.path.join(GOLDEN, f"{name}.npz")) as z:
        return {k: z[k] for k in z.files}


def oracle_observables(g):
    """(CSR, rate) pairs of the fixture's pair projectors embedded at its electron strides."""
    D = g["factors"].shape[0]
    s1, s2 = (int(x) for x in g["electron_strides"])
    idx = np.arange(D)
    d1, d2 = (idx // s1) % 2, (idx // s2) % 2
    base = idx - d1 * s1 - d2 * s2
    out = []
    for op4, rate in zip(g["obs_pair_ops"], g["obs_rates"]):
        A = np.zeros((D, D), np.complex128)
        for a in range(4):
            rows = np.nonzero((2 * d1 + d2) == a)[0]
            for b in range(4):
                if op4[a, b] != 0:
                    A[rows, base[rows] + (b >> 1) * s1 + (b & 1) * s2] += op4[a, b]
        out.append((den.to_csr(A), float(rate)))
    return out


def rel(a, b):
    return np.max(np.abs(np.asarray(a) - np.asarray(b))) / np.max(np.abs(b))


@pytest.mark.parametrize("name", ["plain_small", "st_noise", "dense_branch"])
def test_oracle_reproduces_golden(name):
    g = load(name)
    kw = {}
    if "flip_bits" in g:
        D = g["factors"].shape[0]
        kw = dict(U_csr=orc.st_unitary([2] * int(np.log2(D)), 0, 1), event_rate=0.5 * float(g["st_rate"]),
                  noise_mode=0, seed=float(g["noise_seed"]), seed_mode=0)
    ref = orc.hs_stochastic((g["h_rowptr"], g["h_col"], g["h_val"]), g["factors"], g["times"], oracle_observables(g),
                            kappa=float(g["kappa"]), krylov=int(g["krylov"]),
                            method=1 if name == "dense_branch" else 0, nthreads=4, **kw)
    assert rel(ref["traj_yield"], g["ref_traj_yield"]) < 1e-12
    assert rel(ref["yield"], g["ref_yield"]) < 1e-12
    assert rel(ref["values"], g["ref_values"]) < 1e-12
    assert rel(ref["factors"], g["ref_factors"]) < 1e-12


def test_density_oracle_reproduces_golden():
    g = load("exact_trace")
    D = g["factors"].shape[0]
    H = np.zeros((D, D), np.complex128)
    rows = np.repeat(np.arange(D), np.diff(g["h_rowptr"]))
    H[rows, g["h_col"]] = g["h_val"]
    K = float(g["kappa"]) * np.eye(D)
    ops = [(_dense(op, D), r) for op, r in oracle_observables(g)]
    rho0 = g["factors"] @ g["factors"].conj().T
    values, yields = den.propagate_density(H, K, rho0, g["times"], ops)
    assert rel(values, g["ref_values"]) < 1e-12
    assert rel(yields, g["ref_yield"]) < 1e-12


def _dense(csr, D):
    r, c, v = csr
    A = np.zeros((D, D), np.complex128)
    A[np.repeat(np.arange(D), np.diff(r)), c] = v
    return A


def _same_matrix(csr_a, csr_b, D):
    A, B = _dense(csr_a, D), _dense(csr_b, D)
    return np.max(np.abs(A - B)) / np.max(np.abs(B))


def test_host_assembly_and_samples_reproduce_golden_inputs():
    # plain_small: the plain benchmark system and its trace samples
    g = load("plain_small")
    w = S.plain_small()
    M = g["factors"].shape[1]
    assert _same_matrix(w.system.hamiltonian_csr(), (g["h_rowptr"], g["h_col"], g["h_val"]), w.system.dim) < 1e-14
    assert np.array_equal(w.system.trace_samples(M, w.seed), g["factors"])
    assert np.array_equal(S.time_grid(float(len(g["times"]) - 1), 1.0), g["times"])
    assert tuple(w.system.electron_strides()) == tuple(g["electron_strides"])
    assert w.system.kappa() == float(g["kappa"])
    # st_noise: an anisotropic system, its samples and the reference's flip stream
    g = load("st_noise")
    system = h.random_system([2, 2, 2], [2], seed=11, st_rate=0.05, sink=2e-3, hf_scale=3.0)
    M = g["factors"].shape[1]
    assert _same_matrix(system.hamiltonian_csr(), (g["h_rowptr"], g["h_col"], g["h_val"]), system.dim) < 1e-14
    assert np.array_equal(system.trace_samples(M, float(g["noise_seed"])), g["factors"])
    bits = hs.reference_flip_bits(float(g["noise_seed"]), float(g["st_rate"]), g["times"], M)
    assert np.array_equal(bits, g["flip_bits"])
    assert np.unpackbits(bits).sum() > 20


def test_golden_cases_are_present_and_small():
    for name in CASES:
        path = os.path.join(GOLDEN, f"{name}.npz")
        assert os.path.getsize(path) < 128 * 1024
        g = load(name)
        assert np.all(np.isfinite(g["ref_yield"])) and np.all(g["ref_yield"] > 0)
