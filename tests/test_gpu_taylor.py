"""GPU parity of the Taylor propagator (MSGPU_PROP_TAYLOR, the reference's
propagationmethod=autoexpm, SpinSpace::HighamProp) against the oracle's FP64
expm method: per-trajectory yields within 1e-10 relative at the "double"
tolerance 2^-53, within 1e-6 at the "single" tolerance 2^-24; general
(CSR) K and the reference noise stream included.
"""
import numpy as np
import pytest

from molspin_b200 import _lib as L
from molspin_b200 import hsgeneral as hs
from molspin_b200 import systems as S
from oracle import density as den
from oracle import pyoracle as orc
from tests import helpers as h

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def _taylor(system, F, times, tol=None, K_csr=None, noise=None):
    with hs.HSPropagatorB200(0) as p:
        p.set_hamiltonian(*system.hamiltonian_csr())
        if K_csr is not None:
            p.set_reaction(csr=K_csr)
        else:
            p.set_reaction(kappa=system.kappa())
        p.set_electron_pair(*system.electron_strides())
        p.set_observables([(op, rate) for _, op, rate in system.observables()])
        if noise is not None:
            p.set_noise(*noise)
        if tol is not None:
            p.set_option(L.OPT_TAYLOR_TOL, tol)
        p.set_factors(F)
        p.propagate(times, 16, "c128", propagator="taylor")
        return p.yields()


@pytest.mark.parametrize("tol,bound", [(None, 1e-10), (2.0 ** -24, 1e-6)])
def test_taylor_against_expm_oracle(tol, bound):
    w = S.plain_small()
    M, times = 64, S.time_grid(60.0, 1.0)
    F = w.system.trace_samples(M, w.seed)
    per, ens = _taylor(w.system, F, times, tol)
    ref = orc.hs_stochastic(w.system.hamiltonian_csr(), F, times, h.oracle_observables(w.system),
                            kappa=w.system.kappa(), method=1, nthreads=8)
    assert _rel(per, ref["traj_yield"]) < bound
    assert _rel(ens, ref["yield"]) < bound


def test_taylor_general_K_and_reference_noise():
    system = h.random_system([2, 2], [2, 3], seed=31, st_rate=0.09, hf_scale=2.5)
    system.sinks = {"S": 2e-3, "T0": 1e-3, "Tp": 5e-4, "Tm": 1e-3}  # unequal: K is not a scalar
    K = den.to_csr(sum(0.5 * rate * den.pair_operator(S.pair_projector(S.PAIR_STATES[n]), system)
                       for n, rate in system.sinks.items()), 1e-18)
    M, times = 40, S.time_grid(50.0, 1.0)
    F = system.trace_samples(M, 5.0)
    bits = hs.reference_flip_bits(5.0, system.st_rate, times, M, 0)
    per, _ = _taylor(system, F, times, K_csr=K, noise=(system.st_rate, L.NOISE_REPLAY, 0, bits, len(times) - 1, M))
    ref = orc.hs_stochastic(system.hamiltonian_csr(), F, times, h.oracle_observables(system), K_csr=K, method=1,
                            U_csr=orc.st_unitary(system.mult, *system.electrons), event_rate=0.5 * system.st_rate,
                            noise_mode=1, flip_bits=bits, nthreads=8)
    assert _rel(per, ref["traj_yield"]) < 1e-10


def test_taylor_is_complex128_only():
    w = S.plain_small()
    with hs.HSPropagatorB200(0) as p:
        p.set_hamiltonian(*w.system.hamiltonian_csr())
        p.set_reaction(kappa=w.system.kappa())
        p.set_electron_pair(*w.system.electron_strides())
        p.set_observables([(op, rate) for _, op, rate in w.system.observables()])
        p.set_factors(w.system.trace_samples(8, 1.0))
        with pytest.raises(hs.MsgpuError) as e:
            p.propagate(S.time_grid(3.0, 1.0), 16, "c64", propagator="taylor")
        assert e.value.code == L.MSGPU_ERR_INVALID


@pytest.mark.parametrize("form", ["streamed"])
def test_rk4_against_oracle_restatement(form):
    # the explicit RK4 step (propagationmethod=rk4) against the oracle's RK4,
    # and its fourth-order convergence to the FP64 expm result
    w = S.plain_small()
    M = 32
    F = w.system.trace_samples(M, w.seed)
    errs = []
    for dt in (0.2, 0.1):
        times = S.time_grid(20.0, dt)
        with hs.HSPropagatorB200(0) as p:
            p.set_form(form)
            p.set_hamiltonian(*w.system.hamiltonian_csr())
            p.set_reaction(kappa=w.system.kappa())
            p.set_electron_pair(*w.system.electron_strides())
            p.set_observables([(op, rate) for _, op, rate in w.system.observables()])
            p.set_factors(F)
            p.propagate(times, 16, "c128", propagator="rk4")
            per, _ = p.yields()
        obs = h.oracle_observables(w.system)
        rk = orc.hs_stochastic(w.system.hamiltonian_csr(), F, times, obs, kappa=w.system.kappa(), method=2, nthreads=8)
        ex = orc.hs_stochastic(w.system.hamiltonian_csr(), F, times, obs, kappa=w.system.kappa(), method=1, nthreads=8)
        assert _rel(per, rk["traj_yield"]) < 1e-11
        errs.append(_rel(per, ex["traj_yield"]))
    assert errs[1] < errs[0] / 10  # fourth order: about 16x per halving
