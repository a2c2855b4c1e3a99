"""GPU: time-dependent H through a coefficient schedule (H at each step's
midpoint, as TaskHSGeneral's dynamic loop builds it).

An oscillating field B(t) = B0 z + B1 cos(w t) x: the scheduled run equals
the same steps run one at a time with the coefficients set between them
(bitwise for complex128 Krylov, to rounding for Taylor, to 1e-6 for
complex64), and the oracle driven
step by step with H(t_mid)
(complex128 Krylov and Taylor within 1e-10 per trajectory; reference noise
stream included).
"""
import numpy as np
import pytest

from molspin_b200 import _lib as L
from molspin_b200 import hsgeneral as hs
from molspin_b200 import systems as S
from oracle import pyoracle as orc
from tests import helpers as h

pytestmark = pytest.mark.gpu


def _field(t):
    return np.array([200e-6 * np.cos(0.9 * t), 0.0, 50e-6])


def _system():
    rng = np.random.default_rng(8)
    ta = [S._aniso_tensor(rng, 1.2) for _ in range(3)]
    tb = [S._aniso_tensor(rng, 1.2)]
    s = S.radical_pair([2, 2, 2], [2], ta, tb, np.zeros(3), sink_rate=1e-3, st_rate=0.06)  # D = 64
    return s


def _ctx(p, s, F, r, c, v, noise):
    p.set_form("streamed")
    p.set_hamiltonian_terms(r, c, v, [1.0, 0.0, 0.0, 0.0])
    p.set_reaction(kappa=s.kappa())
    p.set_electron_pair(*s.electron_strides())
    p.set_observables([(op, rate) for _, op, rate in s.observables()])
    p.set_noise(*noise)
    p.set_factors(F)


@pytest.mark.parametrize("precision,propagator", [("c128", "krylov"), ("c64", "krylov"), ("c128", "taylor")])
def test_schedule_equals_stepwise_coefficients(precision, propagator):
    s = _system()
    r, c, v = S.field_terms(s)
    M, times = 32, S.time_grid(24.0, 1.0)
    F = s.trace_samples(M, 4.0)
    mids = 0.5 * (times[1:] + times[:-1])
    coef = np.array([[1.0, *_field(t)] for t in mids])
    noise = (s.st_rate, L.NOISE_PHILOX, 77)
    with hs.HSPropagatorB200(0) as p:
        _ctx(p, s, F, r, c, v, noise)
        p.set_hamiltonian_schedule(coef)
        p.propagate(times, 12, precision, propagator=propagator)
        per_a, _ = p.yields()
        val_a = p.values()
    with hs.HSPropagatorB200(0) as p:
        _ctx(p, s, F, r, c, v, noise)
        vals = []
        for k in range(len(times) - 1):
            p.set_hamiltonian_coefficients(coef[k])
            p.propagate(times[k:k + 2], 12, precision, step_offset=k, accumulate=k > 0, propagator=propagator)
            vals.append(p.values() if k == 0 else p.values()[1:])
        per_b, _ = p.yields()
        val_b = np.concatenate(vals)
    if precision == "c128" and propagator == "krylov":
        np.testing.assert_array_equal(per_a, per_b)
        np.testing.assert_array_equal(val_a, val_b)
    elif propagator == "taylor":
        # the scheduled Taylor step bounds the norm from the terms (possibly
        # another sub-step count): equal to rounding
        np.testing.assert_allclose(per_a, per_b, rtol=1e-13, atol=0)
        np.testing.assert_allclose(val_a, val_b, rtol=1e-13, atol=1e-20)
    else:
        # complex64: every run boundary stores the scaled FP32 state (24 of
        # them here), so the one-step runs agree to the precision form's 1e-6
        np.testing.assert_allclose(per_a, per_b, rtol=1e-6, atol=0)
        np.testing.assert_allclose(val_a, val_b, rtol=1e-6, atol=1e-16)


@pytest.mark.parametrize("propagator", ["krylov", "taylor"])
def test_schedule_against_stepwise_oracle(propagator):
    s = _system()
    r, c, v = S.field_terms(s)
    M, times = 24, S.time_grid(20.0, 1.0)
    F = s.trace_samples(M, 6.0)
    mids = 0.5 * (times[1:] + times[:-1])
    bits = hs.reference_flip_bits(6.0, s.st_rate, times, M, 0)
    with hs.HSPropagatorB200(0) as p:
        _ctx(p, s, F, r, c, v, (s.st_rate, L.NOISE_REPLAY, 0, bits, len(times) - 1, M))
        p.set_hamiltonian_schedule(np.array([[1.0, *_field(t)] for t in mids]))
        p.propagate(times, 16, "c128", propagator=propagator)
        values = p.values()
    # oracle: one step at a time with H(t_mid), this step's two flip halves
    obs = h.oracle_observables(s)
    U = orc.st_unitary(s.mult, *s.electrons)
    allbits = np.unpackbits(bits, bitorder="little")
    state, ref_values = F.copy(), []
    for k in range(len(times) - 1):
        sk = _system()
        sk.linear = []
        S._zeeman(sk, _field(mids[k]))
        step_bits = np.packbits(allbits[2 * k * M:(2 * k + 2) * M], bitorder="little")
        out = orc.hs_stochastic(sk.hamiltonian_csr(), state, times[k:k + 2], obs, kappa=s.kappa(), krylov=16,
                                U_csr=U, event_rate=0.5 * s.st_rate, noise_mode=1, flip_bits=step_bits, nthreads=8)
        ref_values.append(out["values"][0])
        state = out["factors"]
    ref_values.append(out["values"][1])
    ref_values = np.asarray(ref_values)
    assert np.max(np.abs(values - ref_values)) < 1e-10 * np.max(np.abs(ref_values))


def _rk4_rows(times):
    """Coefficient rows of an RK4 schedule: each step's start and midpoint, then the last end."""
    rows = []
    for k in range(len(times) - 1):
        rows.append([1.0, *_field(times[k])])
        rows.append([1.0, *_field(0.5 * (times[k] + times[k + 1]))])
    rows.append([1.0, *_field(times[-1])])
    return np.array(rows)


def test_dynamic_rk4_against_oracle():
    # RK4 with G at each step's start, midpoint and end (StepDynamicRK4Stochastic)
    # against the numpy restatement, replayed noise: within 1e-10
    import scipy.sparse as sp
    from oracle import dynamic as dyn
    s = _system()
    r, c, v = S.field_terms(s)
    D, M = s.dim, 16
    times = S.time_grid(12.0, 0.5)
    F = s.trace_samples(M, 5.0)
    rng = np.random.default_rng(21)
    bits = np.packbits(rng.integers(0, 2, size=2 * (len(times) - 1) * M).astype(np.uint8), bitorder="little")
    with hs.HSPropagatorB200(0) as p:
        _ctx(p, s, F, r, c, v, (s.st_rate, L.NOISE_REPLAY, 0, bits, len(times) - 1, M))
        p.set_hamiltonian_schedule_rk4(_rk4_rows(times))
        p.propagate(times, 12, "c128", propagator="rk4")
        values = p.values()
    terms = [sp.csr_matrix((v[k], c, r), shape=(D, D)).toarray() for k in range(v.shape[0])]

    def H_at(t):
        return sum(ck * T for ck, T in zip([1.0, *_field(t)], terms))

    obs = [(sp.csr_matrix((o[0][2], o[0][1], o[0][0]), shape=(D, D)).toarray(), o[1]) for o in h.oracle_observables(s)]
    ur, uc, uv = orc.st_unitary(s.mult, *s.electrons)
    U = sp.csr_matrix((uv, uc, ur), shape=(D, D)).toarray()
    ref = dyn.dynamic_rk4_stochastic(H_at, s.kappa(), F, times, obs, U, bits)
    assert np.max(np.abs(values - ref)) < 1e-10 * np.max(np.abs(ref))


def test_rk4_schedule_midpoints_drive_krylov_and_rk4_needs_them():
    # the Krylov step reads the midpoint rows of an RK4 schedule: bitwise the
    # run with the midpoint schedule; RK4 with a midpoint-only schedule is refused
    s = _system()
    r, c, v = S.field_terms(s)
    M, times = 16, S.time_grid(8.0, 1.0)
    F = s.trace_samples(M, 7.0)
    mids = 0.5 * (times[1:] + times[:-1])
    noise = (s.st_rate, L.NOISE_PHILOX, 13)
    out = []
    for rk in (False, True):
        with hs.HSPropagatorB200(0) as p:
            _ctx(p, s, F, r, c, v, noise)
            if rk:
                p.set_hamiltonian_schedule_rk4(_rk4_rows(times))
            else:
                p.set_hamiltonian_schedule(np.array([[1.0, *_field(t)] for t in mids]))
            p.propagate(times, 12, "c128")
            out.append(p.values())
            if not rk:
                with pytest.raises(hs.MsgpuError) as e:
                    p.propagate(times, 12, "c128", propagator="rk4")
                assert e.value.code == L.MSGPU_ERR_INVALID
    np.testing.assert_array_equal(out[0], out[1])
