"""Dynamic-H RK4 stochastic loop (numpy, dense, small systems).

TEST INFRASTRUCTURE ONLY: the checker of the device's RK4 propagator with a
time-dependent Hamiltonian.  Restates HSPropagator::StepDynamicRK4Stochastic
(RunSection/General/HS/HSPropagator.cpp:142-150): a half step of the
singlet-triplet noise, then StepDynamicRK4 (:104-128), classical RK4 on
dB/dt = G(t) B with G = -iH(t) - K evaluated at the step's start, midpoint
and end,

    k1 = G0 B, k2 = Gm (B + dt/2 k1), k3 = Gm (B + dt/2 k2), k4 = G1 (B + dt k3),
    B <- B + dt/6 (k1 + 2 k2 + 2 k3 + k4),

then the second noise half step.  The noise halves use replayed bits in the
layout of the C oracle (oracle/hs_oracle.cpp, apply_flips): bit
(2 s + half) M + c, little-endian within each byte.  Observables are
rate * <b|O|b> summed over trajectories at every grid point, as the C
oracle's `values`.
"""
from __future__ import annotations

import numpy as np


def _flip(B: np.ndarray, U: np.ndarray, bits: np.ndarray, s: int, half: int) -> None:
    M = B.shape[1]
    for c in range(M):
        bit = (2 * s + half) * M + c
        if (bits[bit >> 3] >> (bit & 7)) & 1:
            B[:, c] = U @ B[:, c]


def dynamic_rk4_stochastic(H_at, kappa: float, factors: np.ndarray, times, observables, U: np.ndarray,
                           flip_bits: np.ndarray) -> np.ndarray:
    """H_at(t): dense H (rad/ns) at time t; K = kappa I; factors D x M;
    observables: list of (dense O, rate); U: dense singlet-triplet unitary.
    Returns values [ntimes x nobs]."""
    B = np.array(factors, dtype=np.complex128, copy=True)
    D = B.shape[0]
    times = np.asarray(times, dtype=np.float64)
    bits = np.asarray(flip_bits, dtype=np.uint8)
    K = kappa * np.eye(D)

    def evaluate() -> np.ndarray:
        return np.array([rate * np.real(np.sum(np.conj(B) * (O @ B))) for O, rate in observables])

    values = [evaluate()]
    for s in range(len(times) - 1):
        t0, t1 = times[s], times[s + 1]
        dt = t1 - t0
        _flip(B, U, bits, s, 0)
        G0 = -1j * H_at(t0) - K
        Gm = -1j * H_at(t0 + 0.5 * dt) - K
        G1 = -1j * H_at(t1) - K
        k1 = G0 @ B
        k2 = Gm @ (B + 0.5 * dt * k1)
        k3 = Gm @ (B + 0.5 * dt * k2)
        k4 = G1 @ (B + dt * k3)
        B = B + (dt / 6.0) * (k1 + 2.0 * k2 + 2.0 * k3 + k4)
        _flip(B, U, bits, s, 1)
        values.append(evaluate())
    return np.asarray(values)
