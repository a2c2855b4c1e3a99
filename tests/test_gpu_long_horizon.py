"""GPU: accuracy of the reduced-precision forms over long runs, against the
complex128 Krylov path on the same system, trajectories and time grid.

The short parity tests bound one step's error; these bound how it grows over
a full horizon.

- Precision form: complex64 state with FP64 reductions, D=16384, 128
  trajectories, 2000 steps of 0.5 ns.  Measured: per trajectory 8.3e-8,
  ensemble 1.3e-8, the singlet/triplet time series 7.5e-9.
- Dense form, renormalised to the exact survival: D=1024, 64 trajectories,
  20000 steps of 1 ns.  Measured: bf16x3 7.1e-5 per trajectory and 6.0e-5
  ensemble; bf16x6 9.8e-6 and 7.9e-6.  The final norms match complex128
  within 1.2e-7.  Without renormalisation the same runs drift by 7.7 %
  (bf16x3) and 2.6 % (bf16x6) in norm.  The exact-accumulation form int8x4
  (int8 slices, int32 accumulation, FP64 state) is held to the precision
  forms' 1e-6.

Tolerances are about twice the measured errors.
"""
import numpy as np
import pytest

from molspin_b200 import _lib as L
from molspin_b200 import hsgeneral as hs
from molspin_b200 import systems as S

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def _run(system, F, times, krylov, precision, propagator="krylov", renorm=1):
    with hs.HSPropagatorB200(0) as p:
        p.set_hamiltonian(*system.hamiltonian_csr())
        p.set_reaction(kappa=system.kappa())
        p.set_electron_pair(*system.electron_strides())
        p.set_observables([(op, rate) for _, op, rate in system.observables()])
        p.set_option(L.OPT_DENSE_RENORMALIZE, renorm)
        p.set_factors(F)
        p.propagate(times, krylov, precision, propagator=propagator)
        per, ens = p.yields()
        return per, ens, p.values(), p.get_factors()


def test_precision_form_over_2000_steps():
    w = S.precision_large(M=128, steps=2000)
    F = w.system.trace_samples(w.M, w.seed)
    times = w.times()
    per, ens, values, _ = _run(w.system, F, times, w.krylov, "c64")
    per_r, ens_r, values_r, _ = _run(w.system, F, times, w.krylov, "c128")
    assert _rel(per, per_r) < 2e-7
    assert _rel(ens, ens_r) < 3e-8
    assert _rel(values, values_r) < 2e-8


# (precision, per-trajectory tolerance, ensemble tolerance)
# int8x4 (exact int32 accumulation, FP64 state) is held to the precision forms' 1e-6 target
DENSE_TOL = [("bf16x3", 1.5e-4, 1.2e-4), ("bf16x6", 2e-5, 1.6e-5), ("int8x4", 1e-6, 1e-6)]


@pytest.fixture(scope="module")
def dense_reference():
    w = S.dense_tc(M=64, steps=20000)
    F = w.system.trace_samples(w.M, w.seed)
    times = w.times()
    return w, F, times, _run(w.system, F, times, w.krylov, "c128")


@pytest.mark.parametrize("precision,tol_traj,tol_ens", DENSE_TOL)
def test_dense_form_over_20000_steps(dense_reference, precision, tol_traj, tol_ens):
    w, F, times, (per_r, ens_r, values_r, F_r) = dense_reference
    per, ens, values, F_d = _run(w.system, F, times, w.krylov, precision, propagator="dense")
    print(f"{precision}: per-trajectory {_rel(per, per_r):.2e} ensemble {_rel(ens, ens_r):.2e} "
          f"values {_rel(values, values_r):.2e}")
    assert _rel(per, per_r) < tol_traj
    assert _rel(ens, ens_r) < tol_ens
    assert _rel(values, values_r) < tol_ens
    norm_r = np.sum(np.abs(F_r) ** 2, axis=0)
    norm_d = np.sum(np.abs(F_d) ** 2, axis=0)
    assert np.max(np.abs(norm_d - norm_r) / norm_r) < 1e-6
