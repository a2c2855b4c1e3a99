"""GPU: the cluster-resident complex64 Lanczos recurrence (k_lanczos_fused,
MSGPU_OPT_LANCZOS_CLUSTER) against the four-kernel iteration it replaces and
against the complex128 path and the oracle.

The fused kernel applies the same quartet blocks with the same FP32
arithmetic, in stride order instead of neighbour-row order, and sums alpha_j
and |w_{j+1}|^2 in another FP64 order.  Yields of the two complex64 forms
therefore agree to FP32 rounding carried through the run, and both stay within
the precision form's 1e-6 (relative, per trajectory) of complex128.
"""
import numpy as np
import pytest

from molspin_b200 import _lib as L
from molspin_b200 import hsgeneral as hs
from molspin_b200 import systems as S
from oracle import pyoracle as orc
from tests import helpers as h

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def _run(system, F, times, precision, cluster=None, noise=None, krylov=16):
    with hs.HSPropagatorB200(0) as p:
        p.set_form("streamed")
        if cluster is not None:
            p.set_option(L.OPT_LANCZOS_CLUSTER, cluster)
        p.set_hamiltonian(*system.hamiltonian_csr())
        p.set_reaction(kappa=system.kappa())
        p.set_electron_pair(*system.electron_strides())
        p.set_observables([(op, rate) for _, op, rate in system.observables()])
        if noise is not None:
            p.set_noise(*noise)
        p.set_factors(F)
        p.profile(True)
        p.propagate(times, krylov, precision)
        fused = p.profile_read(L.KC_LANCZOS)[1]
        per, ens = p.yields()
        return per, ens, p.values(), fused


@pytest.mark.parametrize("cluster", [1, 2, 4, 8, 16])
def test_cluster_sizes_against_four_kernel_iteration(cluster):
    # D = 1024 (256 quartets over 1..16 CTAs), Philox dephasing, 72
    # trajectories (a padded trajectory block)
    system = h.random_system([2] * 5, [2] * 3, seed=71, aniso=True, st_rate=0.05)
    M, times = 72, S.time_grid(30.0, 1.0)
    F = system.trace_samples(M, 2.0)
    noise = (system.st_rate, L.NOISE_PHILOX, 5)
    per_f, ens_f, val_f, nf = _run(system, F, times, "c64", cluster, noise)
    per_4, ens_4, val_4, n4 = _run(system, F, times, "c64", 0, noise)
    per_d, _, val_d, _ = _run(system, F, times, "c128", None, noise)
    assert nf == len(times) - 1 and n4 == 0
    assert _rel(per_f, per_4) < 1e-6
    assert _rel(val_f, val_4) < 1e-6
    assert _rel(per_f, per_d) < 1e-6
    assert _rel(val_f, val_d) < 1e-6


@pytest.mark.parametrize("cluster", [4, 16])
def test_uneven_split_spin_one_and_interleaved_electrons(cluster):
    # electrons at positions 1 and 3, two spin-1 nuclei: D = 288, 72 quartets;
    # 16 CTAs of 5 quartets leave the last CTA without any
    rng = np.random.default_rng(8)
    s = S.SpinSystem(mult=[2, 2, 3, 2, 2, 3, 2], names=["N1", "E1", "N2", "E2", "N3", "N4", "N5"], electrons=(1, 3))
    for e in (1, 3):
        s.linear.append((e, S.COMMON_PREFACTOR * 2.0023 * 1e-4 * rng.normal(size=3)))
    for e, n in ((1, 0), (1, 2), (3, 4), (3, 5), (1, 6)):
        s.bilinear.append((e, n, S.COMMON_PREFACTOR * 2.0023e-3 * S._aniso_tensor(rng, 2.0)))
    s.sinks = {"S": 2e-3, "T0": 2e-3, "Tp": 2e-3, "Tm": 2e-3}
    s.st_rate = 0.0
    assert s.dim == 288
    M, times = 40, S.time_grid(40.0, 1.0)
    F = rng.normal(size=(s.dim, M)) + 1j * rng.normal(size=(s.dim, M))
    F /= np.linalg.norm(F, axis=0) * np.sqrt(M)
    per_f, _, val_f, nf = _run(s, F, times, "c64", cluster, krylov=12)
    per_4, _, _, _ = _run(s, F, times, "c64", 0, krylov=12)
    ref = orc.hs_stochastic(s.hamiltonian_csr(), F, times, h.oracle_observables(s), kappa=s.kappa(), krylov=12,
                            nthreads=8)
    assert nf == len(times) - 1
    assert _rel(per_f, per_4) < 1e-6
    assert _rel(per_f, ref["traj_yield"]) < 1e-6
    assert _rel(val_f, ref["values"]) < 1e-6


def test_breakdown_in_the_bare_radical_pair():
    # D = 4 with a Krylov dimension above D: the recurrence breaks down and the
    # fused kernel must close T exactly where the four-kernel iteration does
    s = S.radical_pair([], [], [], [], np.array([0.0, 2e-4, 5e-5]), sink_rate=2e-3, st_rate=0.0)
    M, times = 12, S.time_grid(40.0, 1.0)
    F = s.trace_samples(M, 3.0)
    per_f, _, _, nf = _run(s, F, times, "c64", -1, krylov=16)
    per_4, _, _, _ = _run(s, F, times, "c64", 0, krylov=16)
    ref = orc.hs_stochastic(s.hamiltonian_csr(), F, times, h.oracle_observables(s), kappa=s.kappa(), krylov=16)
    assert nf == len(times) - 1
    assert _rel(per_f, per_4) < 1e-6
    assert _rel(per_f, ref["traj_yield"]) < 1e-6


def test_precision_system_block():
    # the D = 16384 precision system (eight CTAs of 512 quartets per cluster)
    w = S.precision_large(M=64, steps=40)
    F = w.system.trace_samples(w.M, w.seed)
    times = w.times()
    per_f, ens_f, val_f, nf = _run(w.system, F, times, "c64", -1, krylov=w.krylov)
    per_4, ens_4, _, n4 = _run(w.system, F, times, "c64", None, krylov=w.krylov)
    per_d, ens_d, _, _ = _run(w.system, F, times, "c128", None, krylov=w.krylov)
    assert nf == len(times) - 1 and n4 == 0
    assert _rel(per_f, per_4) < 1e-6
    assert _rel(per_f, per_d) < 1e-6
    assert _rel(ens_f, ens_d) < 1e-7


def test_option_values():
    with hs.HSPropagatorB200(0) as p:
        for v in (-1, 0, 1, 2, 4, 8, 16):
            p.set_option(L.OPT_LANCZOS_CLUSTER, v)
        for v in (3, 32, -2, 1.5):
            with pytest.raises(hs.MsgpuError):
                p.set_option(L.OPT_LANCZOS_CLUSTER, v)


@pytest.mark.parametrize("noise_mode", ["philox", "replay"])
def test_trajectory_groups_do_not_change_results(noise_mode):
    # MSGPU_OPT_TRAJ_GROUPS: the block in 1, 2 or 4 groups (the second on its
    # own stream) gives bitwise the same yields and values; 1000 trajectories
    # leave the last group partly padded
    system = h.random_system([2] * 5, [2] * 3, seed=72, aniso=True, st_rate=0.06)
    M, times = 1000, S.time_grid(12.0, 1.0)
    F = system.trace_samples(M, 2.5)
    if noise_mode == "philox":
        noise = (system.st_rate, L.NOISE_PHILOX, 17)
    else:
        bits = hs.reference_flip_bits(2.5, system.st_rate, times, M, 0)
        noise = (system.st_rate, L.NOISE_REPLAY, 0, bits, len(times) - 1, M)
    out = {}
    for groups in (1, 2, 4):
        with hs.HSPropagatorB200(0) as p:
            p.set_form("streamed")
            p.set_option(L.OPT_TRAJ_GROUPS, groups)
            p.set_hamiltonian(*system.hamiltonian_csr())
            p.set_reaction(kappa=system.kappa())
            p.set_electron_pair(*system.electron_strides())
            p.set_observables([(op, rate) for _, op, rate in system.observables()])
            p.set_noise(*noise)
            p.set_factors(F)
            p.propagate(times, 12, "c64")
            assert p.get_option(L.OPT_TRAJ_GROUPS) == groups
            out[groups] = (p.yields()[0], p.values(), p.get_factors())
    for groups in (2, 4):
        for a, b in zip(out[groups], out[1]):
            np.testing.assert_array_equal(a, b)
    with hs.HSPropagatorB200(0) as p:
        with pytest.raises(hs.MsgpuError):
            p.set_option(L.OPT_TRAJ_GROUPS, 3)
