"""Generate the golden fixtures of the stochastic HSGeneral path.

Run from the repository root:  python tests/golden/make_golden.py

Every fixture holds the complete inputs of one propagation (H as CSR in
rad/ns, the D x M factor block, the time grid, the reaction rate, the
electron strides, the observables and, where the case has noise, the flip
bits) and the outputs of the CPU oracle for them.  The inputs are built
independently of the product package: H by dense Kronecker products of the
spin matrices (oracle/density.py), the factors by the oracle's restatement of
SpinSpace::BuildTraceSamples (SpinSpace_states.cpp:452-486), the noise bits by
the oracle's restatement of the reference's mt19937 flip stream
(SpinSpace_relaxation.cpp:1201-1254).  The outputs come from the oracle's
restatement of TaskHSGeneral::RunLocal (TaskHSGeneral.cpp:471-560) or, for
the exact-trace case, from the exact density-matrix recursion.

Cases:
  plain_small     the 2e + 4 I=1/2 system of the plain benchmark (D=64,
                  isotropic couplings from seed 0, 50 uT along z, k=1/us),
                  32 trace samples (seed 1), Krylov 16, 200 steps of 1 ns
  st_noise        2e + 3 I=1/2 on A + 1 on B (D=64, anisotropic, seed 11),
                  singlet-triplet dephasing 0.05/ns replayed from the
                  reference's stream (seed 7), 24 samples, Krylov 12,
                  120 steps of 0.5 ns
  exact_trace     2e + 2 I=1/2 on A + 1 on B (D=32, seed 21), the Z=8
                  orthonormal nuclear states as samples, Krylov 16, 80 steps
                  of 1 ns; outputs from the density-matrix oracle
  dense_branch    plain_small's inputs through the dense propagator branch
                  (HSPropagator.cpp:92-100, U = expm(dt G) in FP64), 100 steps
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import density as den  # noqa: E402
from oracle import pyoracle as orc  # noqa: E402

G_E = 2.0023
PREF = 8.79410005e1  # rad ns^-1 T^-1
S2 = 1.0 / math.sqrt(2.0)
SINGLET = np.array([0.0, S2, -S2, 0.0], dtype=np.complex128)
PAIR = {"S": SINGLET, "T0": np.array([0.0, S2, S2, 0.0], np.complex128),
        "Tp": np.array([1.0, 0.0, 0.0, 0.0], np.complex128), "Tm": np.array([0.0, 0.0, 0.0, 1.0], np.complex128)}


class _System:
    """Just the fields the density oracle reads (mult, electrons, linear, bilinear)."""

    def __init__(self, n_a: int, n_b: int):
        self.mult = [2, 2] + [2] * (n_a + n_b)
        self.electrons = (0, 1)
        self.linear = []
        self.bilinear = []
        self.n_a, self.n_b = n_a, n_b

    @property
    def dim(self) -> int:
        return int(np.prod(self.mult))

    def strides(self) -> list[int]:
        return [int(np.prod(self.mult[k + 1:])) for k in range(len(self.mult))]


def _aniso(rng, half_range):
    ev = rng.uniform(-half_range, half_range, size=3)
    q, r = np.linalg.qr(rng.normal(size=(3, 3)))
    q = q * np.sign(np.diag(r))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q @ np.diag(ev) @ q.T


def _radical_pair(couplings_a, couplings_b, field_T):
    s = _System(len(couplings_a), len(couplings_b))
    for e in (0, 1):
        s.linear.append((e, PREF * G_E * np.asarray(field_T, float)))
    for k, a in enumerate(list(couplings_a) + list(couplings_b)):
        e = 0 if k < len(couplings_a) else 1
        A = a * np.eye(3) if np.isscalar(a) else np.asarray(a, float)
        s.bilinear.append((e, 2 + k, PREF * G_E * 1e-3 * A))
    return s


def _observables(system, rate):
    return [(name, den.pair_operator(np.outer(v, v.conj()), system), rate) for name, v in PAIR.items()]


def _common(system, F, times, rate, krylov):
    rowptr, col, val = den.to_csr(den.dense_hamiltonian(system))
    obs = _observables(system, rate)
    return dict(h_rowptr=np.asarray(rowptr, np.int32), h_col=np.asarray(col, np.int32),
                h_val=np.asarray(val, np.complex128), factors=np.asarray(F, np.complex128),
                times=np.asarray(times, np.float64), kappa=np.float64(0.5 * rate), sink_rate=np.float64(rate),
                krylov=np.int32(krylov), electron_strides=np.array([system.dim // 2, system.dim // 4], np.int32),
                obs_names=np.array([n for n, _, _ in obs]), obs_pair_ops=np.array([np.outer(v, v.conj())
                                                                                    for v in PAIR.values()]),
                obs_rates=np.full(len(obs), rate)), [(den.to_csr(op), r) for _, op, r in obs]


def case_plain_small(method=0, steps=200, M=32):
    rng = np.random.default_rng(0)
    a = rng.uniform(-1.0, 1.0, size=4)
    system = _radical_pair(list(a), [], [0.0, 0.0, 50e-6])
    times = orc.time_grid(float(steps), 1.0)
    F = orc.trace_samples(1.0, SINGLET, system.dim // 4, M)
    d, obs = _common(system, F, times, 1e-3, 16)
    ref = orc.hs_stochastic((d["h_rowptr"], d["h_col"], d["h_val"]), F, times, obs, kappa=float(d["kappa"]),
                            krylov=16, method=method, nthreads=8)
    return d, ref


def case_st_noise():
    rng = np.random.default_rng(11)
    dvec = rng.normal(size=3)  # field direction first, then the tensors
    dvec /= np.linalg.norm(dvec)
    ta = [_aniso(rng, 1.5 * 3.0) for _ in range(3)]
    tb = [_aniso(rng, 1.5 * 3.0) for _ in range(1)]
    system = _radical_pair(ta, tb, 0.05e-3 * dvec)
    st_rate, M, seed = 0.05, 24, 7.0
    times = orc.time_grid(60.0, 0.5)
    F = orc.trace_samples(seed, SINGLET, system.dim // 4, M)
    d, obs = _common(system, F, times, 2e-3, 12)
    bits = orc.st_flip_bits(seed, 0, 0, 0.5 * st_rate, times, M)
    U = orc.st_unitary(system.mult, 0, 1)
    ref = orc.hs_stochastic((d["h_rowptr"], d["h_col"], d["h_val"]), F, times, obs, kappa=float(d["kappa"]),
                            krylov=12, U_csr=U, event_rate=0.5 * st_rate, noise_mode=0, seed=seed, seed_mode=0,
                            nthreads=8)
    d.update(st_rate=np.float64(st_rate), noise_seed=np.float64(seed), flip_bits=bits)
    return d, ref


def case_exact_trace():
    rng = np.random.default_rng(21)
    dvec = rng.normal(size=3)  # field direction first, then the tensors
    dvec /= np.linalg.norm(dvec)
    ta = [_aniso(rng, 1.5 * 2.0) for _ in range(2)]
    tb = [_aniso(rng, 1.5 * 2.0) for _ in range(1)]
    system = _radical_pair(ta, tb, 0.05e-3 * dvec)
    times = orc.time_grid(80.0, 1.0)
    F = den.orthonormal_nuclear_samples(system, SINGLET)
    d, _ = _common(system, F, times, 1e-3, 16)
    H = den.dense_hamiltonian(system)
    K = float(d["kappa"]) * np.eye(system.dim)
    ops = [(op, r) for _, op, r in _observables(system, 1e-3)]
    values, yields = den.propagate_density(H, K, den.singlet_density(system), times, ops)
    return d, {"values": values, "yield": yields}


def main() -> None:
    cases = {
        "plain_small": case_plain_small(),
        "st_noise": case_st_noise(),
        "exact_trace": case_exact_trace(),
        "dense_branch": case_plain_small(method=1, steps=100),
    }
    for name, (inputs, ref) in cases.items():
        out = dict(inputs)
        out["ref_values"] = ref["values"]
        out["ref_yield"] = ref["yield"]
        if "traj_yield" in ref:
            out["ref_traj_yield"] = ref["traj_yield"]
            out["ref_factors"] = ref["factors"]
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(f"{name}: D={inputs['factors'].shape[0]} M={inputs['factors'].shape[1]} "
              f"steps={len(inputs['times']) - 1} yields={ref['yield']} -> {os.path.relpath(path, ROOT)} "
              f"({os.path.getsize(path)} bytes)")


if __name__ == "__main__":
    main()
