"""GPU: the cube-blocked quartet SpMMs of the complex64 Lanczos form against
the SIMT quartet SpMM, the complex128 path and the oracle:
- the tensor-core SpMM (k_lanczos_apply_tc, variants 8 and 9: cubes of 16 and
  8 output quartets);
- the TMEM-staged SpMM (k_lanczos_apply_tm, variant 10: persistent CTAs over
  cubes of 8 quartets x 256 trajectories, inputs through TMA, tcgen05.cp and
  tcgen05.ld, FP32 block arithmetic).

All complex64 SpMMs apply the same FP32 quartet blocks; the tensor-core one
splits inputs and blocks into a TF32 head and an FP32 tail and accumulates in
FP32 in tensor memory (dropped products 2^-22 of the result), the TMEM-staged
one sums the same products as the SIMT kernels in another order. Yields of the
complex64 forms agree to FP32 rounding carried through the run and all stay
within the precision form's 1e-6 (relative, per trajectory) of complex128.
"""
import numpy as np
import pytest

from molspin_b200 import _lib as L
from molspin_b200 import hsgeneral as hs
from molspin_b200 import systems as S
from oracle import pyoracle as orc
from tests import helpers as h

pytestmark = pytest.mark.gpu

TC_VARIANTS = [8, 9]   # cube bits 4, 3
TM_VARIANT = 10        # TMEM-staged, cube bits 3
CUBE_VARIANTS = TC_VARIANTS + [TM_VARIANT]
SIMT_VARIANT = 7       # k_lanczos_apply_np<2, 3>


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def _run(system, F, times, precision, variant=None, noise=None, krylov=16):
    with hs.HSPropagatorB200(0) as p:
        p.set_form("streamed")
        if variant is not None:
            p.set_option(L.OPT_SPMM_VARIANT, variant)
        p.set_hamiltonian(*system.hamiltonian_csr())
        p.set_reaction(kappa=system.kappa())
        p.set_electron_pair(*system.electron_strides())
        p.set_observables([(op, rate) for _, op, rate in system.observables()])
        if noise is not None:
            p.set_noise(*noise)
        p.set_factors(F)
        p.profile(True)
        p.propagate(times, krylov, precision)
        napply = p.profile_read(L.KC_APPLY)[1]
        if variant is not None and precision == "c64":
            assert p.spmm_choice()["spmm_variant"] == variant  # the forced SpMM is the one that ran
        per, ens = p.yields()
        return per, ens, p.values(), napply


@pytest.mark.parametrize("variant", CUBE_VARIANTS)
def test_tc_against_simt_and_complex128(variant):
    # D = 1024 (P = 8 quartet bits), anisotropic couplings, Philox dephasing,
    # 200 trajectories (a padded block: the last 56 columns of the tile are zero)
    system = h.random_system([2] * 5, [2] * 3, seed=71, aniso=True, st_rate=0.05)
    M, times = 200, S.time_grid(30.0, 1.0)
    F = system.trace_samples(M, 2.0)
    noise = (system.st_rate, L.NOISE_PHILOX, 5)
    per_t, ens_t, val_t, na = _run(system, F, times, "c64", variant, noise)
    per_s, _, val_s, _ = _run(system, F, times, "c64", SIMT_VARIANT, noise)
    per_d, _, val_d, _ = _run(system, F, times, "c128", None, noise)
    assert na > 0
    assert _rel(per_t, per_s) < 1e-6
    assert _rel(val_t, val_s) < 1e-6
    assert _rel(per_t, per_d) < 1e-6
    assert _rel(val_t, val_d) < 1e-6


def _interleaved(second: int):
    # 8 spin-1/2 spins with electrons at basis positions 1 and `second` (D = 256, P = 6)
    rng = np.random.default_rng(12)
    s = S.SpinSystem(mult=[2] * 8, names=[f"S{i}" for i in range(8)], electrons=(1, second))
    for e in (1, second):
        s.linear.append((e, S.COMMON_PREFACTOR * 2.0023 * 1e-4 * rng.normal(size=3)))
    nuclei = [n for n in range(8) if n not in (1, second)]
    for k, n in enumerate(nuclei):
        e = second if k in (3, 4) else 1
        s.bilinear.append((e, n, S.COMMON_PREFACTOR * 2.0023e-3 * S._aniso_tensor(rng, 2.0)))
    s.sinks = {"S": 2e-3, "T0": 2e-3, "Tp": 2e-3, "Tm": 2e-3}
    assert s.dim == 256
    return s, rng


@pytest.mark.parametrize("variant", CUBE_VARIANTS)
def test_tc_interleaved_electrons_small_tile_against_oracle(variant):
    # electrons at basis positions 1 and 3 (strides 64 and 16: a cube's quartets
    # still have consecutive rows), 64 trajectories: one half-filled 128-trajectory tile
    s, rng = _interleaved(3)
    M, times = 64, S.time_grid(40.0, 1.0)
    F = rng.normal(size=(s.dim, M)) + 1j * rng.normal(size=(s.dim, M))
    F /= np.linalg.norm(F, axis=0) * np.sqrt(M)
    per_t, _, val_t, _ = _run(s, F, times, "c64", variant, krylov=12)
    ref = orc.hs_stochastic(s.hamiltonian_csr(), F, times, h.oracle_observables(s), kappa=s.kappa(), krylov=12,
                            nthreads=8)
    assert _rel(per_t, ref["traj_yield"]) < 1e-6
    assert _rel(val_t, ref["values"]) < 1e-6


@pytest.mark.parametrize("variant", [8, TM_VARIANT])
def test_tc_precision_configuration_two_groups(variant):
    # D = 16384 (P = 12), 512 trajectories: two trajectory groups of 256 on two
    # streams; 100 steps against the SIMT SpMM and complex128
    w = S.precision_large(M=512, steps=100)
    F = w.system.trace_samples(w.M, w.seed)
    times = w.times()
    per_t, ens_t, val_t, _ = _run(w.system, F, times, "c64", variant, krylov=w.krylov)
    per_s, _, _, _ = _run(w.system, F, times, "c64", SIMT_VARIANT, krylov=w.krylov)
    per_d, ens_d, val_d, _ = _run(w.system, F, times, "c128", krylov=w.krylov)
    assert _rel(per_t, per_s) < 1e-6
    assert _rel(per_t, per_d) < 1e-6
    assert np.max(np.abs(ens_t - ens_d) / np.abs(ens_d)) < 1e-6
    assert _rel(val_t, val_d) < 1e-6


@pytest.mark.parametrize("variant", [8, TM_VARIANT])
def test_tc_tables_follow_field_terms(variant):
    # H = H_0 + Bx Zx + By Zy + Bz Zz: a field change through the coefficients
    # refreshes the tensor-core tables on the device; the result equals the
    # complex128 path of a context built for the new field
    rng = np.random.default_rng(33)
    ta = [S._aniso_tensor(rng, 1.5) for _ in range(4)]
    tb = [S._aniso_tensor(rng, 1.5) for _ in range(3)]

    def pair(B):
        return S.radical_pair([2] * 4, [2] * 3, ta, tb, np.asarray(B), sink_rate=1e-3)  # D = 512

    B1 = np.array([0.0, 0.0, 50e-6])
    d = np.array([0.3, -0.5, 0.81])
    B2 = 80e-6 * d / np.linalg.norm(d)
    s1 = pair(B1)
    r, c, v = S.field_terms(s1)
    M, times = 128, S.time_grid(40.0, 1.0)
    F = s1.trace_samples(M, 2.0)
    with hs.HSPropagatorB200(0) as p:
        p.set_form("streamed")
        p.set_option(L.OPT_SPMM_VARIANT, variant)
        p.set_hamiltonian_terms(r, c, v, [1.0, *B1])
        p.set_reaction(kappa=s1.kappa())
        p.set_electron_pair(*s1.electron_strides())
        p.set_observables([(op, rate) for _, op, rate in s1.observables()])
        p.set_factors(F)
        p.propagate(times, 14, "c64")
        per1, _ = p.yields()
        p.set_hamiltonian_coefficients([1.0, *B2])
        p.set_factors(F)
        p.propagate(times, 14, "c64")
        per2, _ = p.yields()
    for B, per in ((B1, per1), (B2, per2)):
        ref, _, _, _ = _run(pair(B), F, times, "c128", krylov=14)
        assert _rel(per, ref) < 1e-6
    assert _rel(per1, per2) > 1e-4


def test_tm_second_electron_stride_of_one_cube_against_oracle():
    # electrons at positions 1 and 4: the second stride is 8, one 8-quartet cube,
    # so the TMEM-staged SpMM's boxes still load whole cubes; 320 trajectories:
    # a full and a partly filled 256-trajectory tile
    s, rng = _interleaved(4)
    M, times = 320, S.time_grid(30.0, 1.0)
    F = rng.normal(size=(s.dim, M)) + 1j * rng.normal(size=(s.dim, M))
    F /= np.linalg.norm(F, axis=0) * np.sqrt(M)
    per_t, _, val_t, _ = _run(s, F, times, "c64", TM_VARIANT, krylov=12)
    ref = orc.hs_stochastic(s.hamiltonian_csr(), F, times, h.oracle_observables(s), kappa=s.kappa(), krylov=12,
                            nthreads=8)
    assert _rel(per_t, ref["traj_yield"]) < 1e-6
    assert _rel(val_t, ref["values"]) < 1e-6


@pytest.mark.parametrize("variant", CUBE_VARIANTS)
def test_tc_refused_without_the_nuclear_bit_structure(variant):
    # a spin-1 nucleus: quartets are not bit-indexed, so the forced cube-blocked
    # variant is refused with an error rather than run
    s = h.random_system([2, 3], [2], seed=3)
    F = s.trace_samples(64, 1.0)
    with pytest.raises(hs.MsgpuError):
        _run(s, F, S.time_grid(4.0, 1.0), "c64", variant)


def test_tc_refused_when_a_cube_is_not_consecutive_rows():
    # electrons at positions 1 and 4: the second stride is 8, so a 16-quartet
    # cube's rows are not consecutive and variant 8's boxes cannot load it
    s, rng = _interleaved(4)
    F = rng.normal(size=(s.dim, 64)) + 1j * rng.normal(size=(s.dim, 64))
    F /= np.linalg.norm(F, axis=0) * 8.0
    with pytest.raises(hs.MsgpuError):
        _run(s, F, S.time_grid(4.0, 1.0), "c64", 8)
