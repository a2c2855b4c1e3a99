"""GPU: Hamiltonian as fixed-pattern terms, H = H_0 + Bx Zx + By Zy + Bz Zz
(msgpu_upload_hamiltonian_terms / msgpu_set_hamiltonian_coefficients).

A context that changes the field direction through the coefficients must give
the same yields as a fresh context built for that field: per trajectory within
1e-12 relative in complex128 (the combined H differs from the directly built
one only in summation order), within 1e-7 in complex64 and 1e-6 in the dense
bf16x6 form (the same H rounded the same way, structure built once).
"""
import numpy as np
import pytest

from molspin_b200 import hsgeneral as hs
from molspin_b200 import systems as S

pytestmark = pytest.mark.gpu


def _pair(B):
    rng = np.random.default_rng(33)
    ta = [S._aniso_tensor(rng, 1.5) for _ in range(4)]
    tb = [S._aniso_tensor(rng, 1.5) for _ in range(3)]
    return S.radical_pair([2] * 4, [2] * 3, ta, tb, np.asarray(B), sink_rate=1e-3)  # D = 512


def _setup(p, system, F):
    p.set_reaction(kappa=system.kappa())
    p.set_electron_pair(*system.electron_strides())
    p.set_observables([(op, rate) for _, op, rate in system.observables()])
    p.set_factors(F)


def _rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


@pytest.mark.parametrize("precision,propagator,tol", [("c128", "krylov", 1e-12), ("c64", "krylov", 1e-7),
                                                      ("bf16x6", "dense", 1e-6)])
def test_field_change_through_coefficients(precision, propagator, tol):
    B1 = np.array([0.0, 0.0, 50e-6])
    d = np.array([0.3, -0.5, 0.81])
    B2 = 80e-6 * d / np.linalg.norm(d)
    s1 = _pair(B1)
    r, c, v = S.field_terms(s1)
    M, times = 48, S.time_grid(40.0, 1.0)
    F = s1.trace_samples(M, 2.0)
    with hs.HSPropagatorB200(0) as p:
        p.set_form("streamed")
        p.set_hamiltonian_terms(r, c, v, [1.0, *B1])
        _setup(p, s1, F)
        p.propagate(times, 14, precision, propagator=propagator)
        per1, _ = p.yields()
        p.set_hamiltonian_coefficients([1.0, *B2])
        p.set_factors(F)
        p.propagate(times, 14, precision, propagator=propagator)
        per2, _ = p.yields()
    for B, per in ((B1, per1), (B2, per2)):
        direct = _pair(B)
        with hs.HSPropagatorB200(0) as q:
            q.set_form("streamed")
            q.set_hamiltonian(*direct.hamiltonian_csr())
            _setup(q, direct, F)
            q.propagate(times, 14, precision, propagator=propagator)
            ref, _ = q.yields()
        assert _rel(per, ref) < tol
    assert _rel(per1, per2) > 1e-4  # the field change is visible


def test_coefficients_need_terms():
    s1 = _pair([0.0, 0.0, 50e-6])
    with hs.HSPropagatorB200(0) as p:
        p.set_hamiltonian(*s1.hamiltonian_csr())
        with pytest.raises(hs.MsgpuError):
            p.set_hamiltonian_coefficients([1.0, 0.0, 0.0, 1e-4])


def test_powder_loop_matches_one_context_per_orientation():
    # the orientation loop on one context (field through the coefficients)
    # against a freshly built system per orientation, reference noise stream
    base = _pair([0.0, 0.0, 0.0])
    base.st_rate = 0.05
    grid = S.sphere_grid(4)
    plan = hs.HSExecutionPlan(totaltime=30.0, timestep=1.0, krylovsize=12, montecarlosamples=24, seed=3.0)
    out = hs.run_powder_yields(base, plan, 50e-6, grid)
    ref = []
    for i, d in enumerate(grid):
        s = _pair(50e-6 * d)
        s.st_rate = 0.05
        ref.append(hs.run_stochastic_yields(s, plan, orientation=i)["yields"])
    ref = np.asarray(ref)
    assert _rel(out["orientation_yields"], ref) < 1e-12
    assert _rel(out["yields"], ref.mean(axis=0)) < 1e-12
