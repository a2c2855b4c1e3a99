"""GPU parity against the committed golden fixtures (tests/golden/*.npz).

Each case feeds the fixture's own inputs (H as CSR, factors, time grid,
reaction rate, electron strides, pair observables, replayed flip bits)
through the C ABI and compares with the outputs stored beside them.
Tolerances: complex128 Krylov and Taylor within 1e-10 relative (per
trajectory, ensemble, observable rows and final factors); complex64 within
1e-6; the split-BF16 dense propagator (bf16x6) within 1e-5 per trajectory
and 5e-6 for the ensemble.
"""
import numpy as np
import pytest

from molspin_b200 import _lib as L
from molspin_b200 import hsgeneral as hs
from tests.test_golden import load, rel

pytestmark = pytest.mark.gpu


def run(g, precision="c128", form="auto", propagator="krylov", krylov=None):
    with hs.HSPropagatorB200(0) as p:
        p.set_form(form)
        p.set_hamiltonian(g["h_rowptr"], g["h_col"], g["h_val"])
        p.set_reaction(kappa=float(g["kappa"]))
        p.set_electron_pair(*(int(x) for x in g["electron_strides"]))
        p.set_observables(list(zip(g["obs_pair_ops"], (float(r) for r in g["obs_rates"]))))
        if "flip_bits" in g:
            M = g["factors"].shape[1]
            p.set_noise(float(g["st_rate"]), L.NOISE_REPLAY, 0, g["flip_bits"], len(g["times"]) - 1, M)
        p.set_factors(g["factors"])
        p.propagate(g["times"], int(g["krylov"]) if krylov is None else krylov, precision, propagator=propagator)
        per, ens = p.yields()
        return per, ens, p.values(), p.get_factors()


@pytest.mark.parametrize("name", ["plain_small", "st_noise"])
@pytest.mark.parametrize("form", ["streamed", "resident"])
def test_complex128_matches_golden(name, form):
    g = load(name)
    per, ens, values, F = run(g, form=form)
    assert rel(per, g["ref_traj_yield"]) < 1e-10
    assert rel(ens, g["ref_yield"]) < 1e-10
    assert rel(values, g["ref_values"]) < 1e-10
    assert rel(F, g["ref_factors"]) < 1e-10


@pytest.mark.parametrize("form", ["streamed", "resident"])
def test_complex64_matches_golden(form):
    g = load("plain_small")
    per, ens, _, _ = run(g, precision="c64", form=form)
    assert rel(per, g["ref_traj_yield"]) < 1e-6
    assert rel(ens, g["ref_yield"]) < 1e-6


def test_exact_trace_matches_density_golden():
    g = load("exact_trace")
    _, ens, values, _ = run(g)
    assert rel(ens, g["ref_yield"]) < 1e-10
    assert rel(values, g["ref_values"]) < 1e-10


def test_dense_branch_golden():
    g = load("dense_branch")
    # the reference's autoexpm method at its double tolerance reproduces exp(dt G)
    per, ens, _, _ = run(g, propagator="taylor")
    assert rel(per, g["ref_traj_yield"]) < 1e-10
    assert rel(ens, g["ref_yield"]) < 1e-10
    # the tensor-core propagator, six split-BF16 products
    per, ens, values, _ = run(g, precision="bf16x6", propagator="dense")
    assert rel(per, g["ref_traj_yield"]) < 1e-5
    assert rel(ens, g["ref_yield"]) < 5e-6
    assert rel(values, g["ref_values"]) < 1e-5
