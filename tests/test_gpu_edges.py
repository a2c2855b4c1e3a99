"""GPU edge cases against the oracle (complex128, per-trajectory yields within
1e-10 relative unless stated): a single time point (no step), one
trajectory, the bare radical pair (D = 4, no nuclei), a Krylov dimension
above D, a non-uniform exact-endpoint grid (the last interval shorter), a
zero dephasing rate (no draws, no flips), and a run of one step.
"""
import numpy as np
import pytest

from molspin_b200 import _lib as L
from molspin_b200 import hsgeneral as hs
from molspin_b200 import systems as S
from oracle import pyoracle as orc
from tests import helpers as h

pytestmark = pytest.mark.gpu

FORMS = ["streamed", "resident"]


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def _run(system, F, times, krylov=16, form="auto", noise=None, precision="c128"):
    with hs.HSPropagatorB200(0) as p:
        p.set_form(form)
        p.set_hamiltonian(*system.hamiltonian_csr())
        p.set_reaction(kappa=system.kappa())
        p.set_electron_pair(*system.electron_strides())
        p.set_observables([(op, rate) for _, op, rate in system.observables()])
        if noise is not None:
            p.set_noise(*noise)
        p.set_factors(F)
        p.propagate(times, krylov, precision)
        per, ens = p.yields()
        return per, ens, p.values(), p.get_factors()


def _oracle(system, F, times, krylov=16, **kw):
    return orc.hs_stochastic(system.hamiltonian_csr(), F, times, h.oracle_observables(system), kappa=system.kappa(),
                             krylov=krylov, nthreads=8, **kw)


@pytest.mark.parametrize("form", FORMS)
def test_single_time_point_evaluates_only(form):
    s = h.random_system([2, 2], [2], seed=61)
    F = s.trace_samples(10, 1.0)
    per, ens, values, Fg = _run(s, F, np.array([0.0]), form=form)
    ref = _oracle(s, F, np.array([0.0]))
    assert np.all(per == 0.0) and np.all(ens == 0.0)  # no interval, no yield
    assert _rel(values, ref["values"]) < 1e-12
    assert np.max(np.abs(Fg - F)) == 0.0  # the state is untouched


@pytest.mark.parametrize("form", FORMS)
def test_one_trajectory_and_one_step(form):
    s = h.random_system([2, 3], [2], seed=62)
    F = s.trace_samples(1, 2.0)
    for times in (S.time_grid(1.0, 1.0), S.time_grid(25.0, 1.0)):
        per, ens, _, _ = _run(s, F, times, form=form)
        ref = _oracle(s, F, times)
        assert _rel(per, ref["traj_yield"]) < 1e-10


@pytest.mark.parametrize("form", FORMS)
def test_bare_radical_pair_and_krylov_above_dimension(form):
    # D = 4: two electrons only; krylov 16 > D is capped at D (exact Krylov space)
    s = S.radical_pair([], [], [], [], np.array([0.0, 2e-4, 5e-5]), sink_rate=2e-3, st_rate=0.1)
    assert s.dim == 4
    F = s.trace_samples(12, 3.0)
    times = S.time_grid(40.0, 1.0)
    bits = hs.reference_flip_bits(3.0, s.st_rate, times, 12, 0)
    per, _, _, _ = _run(s, F, times, krylov=16, form=form, noise=(s.st_rate, L.NOISE_REPLAY, 0, bits, len(times) - 1, 12))
    ref = _oracle(s, F, times, krylov=16, U_csr=orc.st_unitary(s.mult, 0, 1), event_rate=0.5 * s.st_rate,
                  noise_mode=1, flip_bits=bits)
    assert _rel(per, ref["traj_yield"]) < 1e-10


def test_exact_endpoint_grid_with_a_short_last_interval():
    s = h.random_system([2, 2], [2, 2], seed=63)
    F = s.trace_samples(20, 4.0)
    times = S.time_grid(10.3, 1.0)  # 0, 1, ..., 10, 10.3
    assert abs((times[-1] - times[-2]) - 0.3) < 1e-12
    for form in FORMS:
        per, _, values, _ = _run(s, F, times, form=form)
        ref = _oracle(s, F, times)
        assert _rel(per, ref["traj_yield"]) < 1e-10
        assert _rel(values, ref["values"]) < 1e-10


def test_zero_dephasing_rate_draws_nothing():
    s = h.random_system([2, 2], [2], seed=64, st_rate=0.0)
    F = s.trace_samples(16, 5.0)
    times = S.time_grid(20.0, 1.0)
    bits = hs.reference_flip_bits(5.0, 0.0, times, 16, 0)
    assert not bits.any()
    a = _run(s, F, times, noise=(0.0, L.NOISE_PHILOX, 11))
    b = _run(s, F, times)
    np.testing.assert_array_equal(a[0], b[0])
