"""GPU: the benchmark configurations at their configured sizes, through the C ABI.

- Plain small configuration (2 electrons + 4 nuclei, D=64, 256 trajectories,
  5000 steps of 1 ns, Krylov dimension 16, complex128): per-trajectory
  singlet yields within 1e-10 (relative) of the oracle's, which is the CPU
  restatement of HSGeneral's per-column Krylov loop, on the same
  trace-sampled factors; streamed and resident forms.
- Precision configuration (D=16384, m=20, dt 0.5 ns): the complex64 form
  against the complex128 form over 5000 steps on a 64-trajectory slice of
  the configured block; per-trajectory and ensemble yields and the
  population time series within 1e-6 (the precision form's target).
"""
import os

import numpy as np
import pytest

from molspin_b200 import hsgeneral as hs
from molspin_b200 import systems as S
from oracle import pyoracle as orc
from tests import helpers as h

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def _run(system, F, times, krylov, precision, form="auto"):
    with hs.HSPropagatorB200(0) as p:
        p.set_form(form)
        p.set_hamiltonian(*system.hamiltonian_csr())
        p.set_reaction(kappa=system.kappa())
        p.set_electron_pair(*system.electron_strides())
        p.set_observables([(op, rate) for _, op, rate in system.observables()])
        p.set_factors(F)
        p.propagate(times, krylov, precision)
        per, ens = p.yields()
        return per, ens, p.values()


@pytest.fixture(scope="module")
def config1_oracle():
    w = S.plain_small()
    assert (w.system.dim, w.M, w.steps, w.krylov) == (64, 256, 5000, 16)
    F = w.system.trace_samples(w.M, w.seed)
    times = w.times()
    assert len(times) == 5001
    ref = orc.hs_stochastic(w.system.hamiltonian_csr(), F, times, h.oracle_observables(w.system),
                            kappa=w.system.kappa(), krylov=w.krylov, nthreads=os.cpu_count() or 1)
    return w, F, times, ref


@pytest.mark.parametrize("form", ["streamed", "resident"])
def test_config1_full_size_per_trajectory(config1_oracle, form):
    w, F, times, ref = config1_oracle
    per, ens, values = _run(w.system, F, times, w.krylov, "c128", form=form)
    assert per.shape == ref["traj_yield"].shape == (256, 4)
    assert _rel(per, ref["traj_yield"]) < 1e-10
    assert np.max(np.abs(ens - ref["yield"]) / np.abs(ref["yield"])) < 1e-10
    assert _rel(values, ref["values"]) < 1e-10


def test_config2_c64_against_c128_over_5000_steps():
    w = S.precision_large(M=1024, steps=5000)
    F = np.ascontiguousarray(w.system.trace_samples(w.M, w.seed)[:, :64])  # a slice of the configured block
    times = w.times()
    assert len(times) == 5001 and w.system.dim == 16384 and w.krylov == 20
    per, ens, values = _run(w.system, F, times, w.krylov, "c64")
    per_r, ens_r, values_r = _run(w.system, F, times, w.krylov, "c128")
    assert _rel(per, per_r) < 1e-6
    assert np.max(np.abs(ens - ens_r) / np.abs(ens_r)) < 1e-6
    assert _rel(values, values_r) < 1e-6
