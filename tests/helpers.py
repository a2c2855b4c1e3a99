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


# The reference's recorded result for its input-file example
# Tests/StochasticRelaxation/st_dephasing.msd (8192 samples, seed 431, dt 0.025 ns over 2 ns):
# max |stochastic - direct| population difference over the 81 x 4 data-file values
# (RunSection/General/HS/STOCHASTIC_RELAXATION.md:250-251), printed to 8 significant digits.
ST_DEPHASING_POPULATION_ERROR = 0.0012766377
# Tolerance: half a unit of the recorded figure's last digit plus the propagators'
# own differences (every one of the reference's propagators records 0.00127664, :236).
ST_DEPHASING_PIN_TOL = 1e-10


def st_dephasing_direct(system, times):
    """The example's "direct" task (sampling=direct; propagationmethod=rk4) on the same grid:
    density-matrix RK4 with the ST dephasing Operator; S, T0, T+, T- populations."""
    H = den.dense_hamiltonian(system)
    K = 0.5 * system.sinks["S"] * np.eye(system.dim)
    ops = [(den.pair_operator(S.pair_projector(S.PAIR_STATES[n]), system), 1.0) for n in ("S", "T0", "Tp", "Tm")]
    return den.st_dephasing_rk4(H, K, den.singlet_density(system), times, ops, den.st_unitary(system),
                                system.st_rate)
