"""Shared fixtures for the tests: small radical-pair systems and their oracle inputs."""
from __future__ import annotations

import math

import numpy as np

from molspin_b200 import systems as S
from oracle import density as den


def st_fixture(field: bool = True, nucleus: bool = True, st_rate: float = 0.7, sink: float = 0.2) -> S.SpinSystem:
    """The reference's st_relaxation_tests::Fixture (Tests/tests_StochasticRelaxation.cpp:133-159):
    E1, E2 and an uncoupled spin-1/2 N; four sinks (S, T0, T+, T-) with rate 0.2;
    H = 0.8 Sz(E1) (commonprefactor=false, prefactor=1); ST dephasing rate 0.7."""
    mult = [2, 2] + ([2] if nucleus else [])
    names = ["E1", "E2"] + (["N"] if nucleus else [])
    s = S.SpinSystem(mult=mult, names=names, electrons=(0, 1))
    if field:
        s.linear.append((0, np.array([0.0, 0.0, 0.8])))
    s.sinks = {"S": sink, "T0": sink, "Tp": sink, "Tm": sink}
    s.st_rate = st_rate
    return s


def random_system(n_a: list[int], n_b: list[int], seed: int, aniso: bool = True, field_mT: float = 0.05,
                  sink: float = 1e-3, st_rate: float = 0.0, hf_scale: float = 1.0) -> S.SpinSystem:
    rng = np.random.default_rng(seed)

    def coup(n):
        return [S._aniso_tensor(rng, 1.5 * hf_scale) if aniso else rng.uniform(-hf_scale, hf_scale) for _ in n]

    d = rng.normal(size=3)
    d /= np.linalg.norm(d)
    return S.radical_pair(n_a, n_b, coup(n_a), coup(n_b), field_mT * 1e-3 * d, sink_rate=sink, st_rate=st_rate)


def oracle_observables(system: S.SpinSystem):
    """Transition observables as (CSR, rate) for the oracle."""
    out = []
    for _, op, rate in system.observables():
        out.append((den.to_csr(den.pair_operator(op, system)), rate))
    return out


def state_population_observables(system: S.SpinSystem):
    """State populations (rate 1) of S, T0, T+, T- for time-evolution checks."""
    out = []
    for name in ("S", "T0", "Tp", "Tm"):
        op = S.pair_projector(S.PAIR_STATES[name])
        out.append((den.to_csr(den.pair_operator(op, system)), 1.0))
    return out


def dense_csr(system: S.SpinSystem):
    return den.to_csr(den.dense_hamiltonian(system))


def survival_bound():
    return 2e-6


def six_sigma(M: int) -> float:
    return 6.0 / (2.0 * math.sqrt(M))
