"""Radical-pair spin systems for the HSGeneral stochastic path.

A :class:`SpinSystem` is the subset of MolSpin's SpinAPI object model that the
hot path needs: spins (multiplicities, in basis order), linear terms
``w . S_k`` and bilinear terms ``S_i^T C S_j`` already converted to rad/ns,
the two radical-pair electrons carrying the singlet-triplet structure, sink
rates and the singlet-triplet dephasing rate.

Unit conventions follow the reference:
  * common prefactor mu_B/hbar = 8.79410005e1 rad ns^-1 T^-1
    (SpinAPI/SpinSpace/SpinSpace_hamiltonians.cpp:747-748);
  * Zeeman ``S . (G . B)`` with the spin's tensor G (isotropic g for the
    electrons, Spin.cpp:29 default 2.0), field in T
    (SpinSpace_hamiltonians.cpp:450-480);
  * hyperfine as in the MolSpin examples (Example/magnetoreception/
    quantumyield_standard/example_2.msd:51-69): interaction prefactor 0.001
    (mT -> T), ``ignoretensors`` unset, so the coupling is
    ``T_e . T_n = g_e S_e^T A I_n`` with A in mT held as the nucleus tensor
    (Spin::Tx/Ty/Tz, Spin.cpp:360-410; SpinSpace_hamiltonians.cpp:481-535);
  * rates in 1/ns, times in ns.

The synthetic generators reproduce the shapes and value distributions of the
benchmark configurations with seeded numpy generators (no external data).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

COMMON_PREFACTOR = 8.79410005e1  # rad ns^-1 T^-1
G_ELECTRON = 2.0023

# Pair-basis projectors (basis |e1 e2> = uu, ud, du, dd; digit 0 = m=+1/2).
_s = 1.0 / math.sqrt(2.0)
SINGLET = np.array([0.0, _s, -_s, 0.0], dtype=np.complex128)
T0 = np.array([0.0, _s, _s, 0.0], dtype=np.complex128)
TPLUS = np.array([1.0, 0.0, 0.0, 0.0], dtype=np.complex128)
TMINUS = np.array([0.0, 0.0, 0.0, 1.0], dtype=np.complex128)
PAIR_STATES = {"S": SINGLET, "T0": T0, "Tp": TPLUS, "Tm": TMINUS}


def pair_projector(v: np.ndarray) -> np.ndarray:
    return np.outer(v, v.conj())


@dataclass
class SpinSystem:
    mult: list[int]                                   # multiplicities, basis order
    names: list[str]
    electrons: tuple[int, int] = (0, 1)               # radical-pair electrons
    linear: list[tuple[int, np.ndarray]] = field(default_factory=list)           # (spin, w[3]) rad/ns
    bilinear: list[tuple[int, int, np.ndarray]] = field(default_factory=list)    # (i, j, C[3,3]) rad/ns
    sinks: dict[str, float] = field(default_factory=dict)                        # pair state -> rate 1/ns
    st_rate: float = 0.0                                                          # dephasing Operator rate 1/ns

    @property
    def dim(self) -> int:
        return int(np.prod(self.mult))

    def strides(self) -> list[int]:
        s, out = 1, [0] * len(self.mult)
        for k in range(len(self.mult) - 1, -1, -1):
            out[k] = s
            s *= self.mult[k]
        return out

    def electron_strides(self) -> tuple[int, int]:
        st = self.strides()
        return st[self.electrons[0]], st[self.electrons[1]]

    def kappa(self) -> float:
        """K = sum_c k_c/2 P_c; a scalar when all four pair sinks share one rate."""
        rates = set(self.sinks.get(k, 0.0) for k in ("S", "T0", "Tp", "Tm"))
        if len(rates) != 1:
            raise ValueError("reaction operator is not a scalar (unequal sinks)")
        return 0.5 * rates.pop()

    def observables(self) -> list[tuple[str, np.ndarray, float]]:
        """Transition-yield observables rate * P_source, in sink order."""
        return [(name, pair_projector(PAIR_STATES[name]), rate) for name, rate in self.sinks.items()]

    # ------------------------------------------------------------ host builder
    def hamiltonian_csr(self):
        """H in rad/ns as CSR (rowptr int32, col int32, val complex128)."""
        from . import _lib as L
        mult = np.asarray(self.mult, dtype=np.int32)
        lin_spin = np.asarray([k for k, _ in self.linear], dtype=np.int32)
        lin_w = np.ascontiguousarray(np.array([w for _, w in self.linear], dtype=np.float64).reshape(-1))
        bi = np.asarray([i for i, _, _ in self.bilinear], dtype=np.int32)
        bj = np.asarray([j for _, j, _ in self.bilinear], dtype=np.int32)
        bc = np.ascontiguousarray(np.array([c for _, _, c in self.bilinear], dtype=np.float64).reshape(-1))
        args = (len(self.mult), L.iptr(mult), len(self.linear), L.iptr(lin_spin) if len(lin_spin) else None,
                L.dptr(lin_w) if len(lin_w) else None, len(self.bilinear), L.iptr(bi) if len(bi) else None,
                L.iptr(bj) if len(bj) else None, L.dptr(bc) if len(bc) else None)
        nnz = L.lib.msgpu_host_build_hamiltonian(*args, None, None, None)
        if nnz < 0:
            raise ValueError("invalid spin system for Hamiltonian assembly")
        D = self.dim
        rowptr = np.zeros(D + 1, dtype=np.int32)
        col = np.zeros(max(1, nnz), dtype=np.int32)
        val = np.zeros(max(1, nnz), dtype=np.complex128)
        L.lib.msgpu_host_build_hamiltonian(*args, L.iptr(rowptr), L.iptr(col), L.dptr(val.view(np.float64)))
        return rowptr, col[:nnz], val[:nnz]

    def trace_samples(self, M: int, seed: float, state: str = "S") -> np.ndarray:
        """SU(Z) trace samples |psi_pair> x chi_j / sqrt(M), D x M column-major
        (reference fast path; requires the electrons to be the leading spins)."""
        if tuple(self.electrons) != (0, 1):
            raise ValueError("the tensor fast path needs the radical pair as the two leading spins")
        from . import _lib as L
        F, Z = 4, self.dim // 4
        fixed = np.ascontiguousarray(PAIR_STATES[state])
        out = np.zeros((M, self.dim), dtype=np.complex128)  # row t = column t of the D x M matrix
        rc = L.lib.msgpu_host_trace_samples(float(seed), L.dptr(fixed.view(np.float64)), F, Z, M,
                                            L.dptr(out.view(np.float64)))
        if rc:
            raise ValueError("trace sampling failed")
        return out.T  # D x M view (Fortran order)


# ------------------------------------------------------------------ builders
def _zeeman(sys_: SpinSystem, field_T: np.ndarray, g: float = G_ELECTRON):
    for e in sys_.electrons:
        sys_.linear.append((e, COMMON_PREFACTOR * g * np.asarray(field_T, dtype=np.float64)))


def field_terms(system: SpinSystem):
    """H(B) = H_0 + Bx Z_x + By Z_y + Bz Z_z (B in T) on one CSR pattern.

    H_0 is the system without its linear (Zeeman) terms, Z_a the electron
    Zeeman operator of a 1 T field along axis a (g = 2.0023, as radical_pair
    builds it).  Returns (rowptr, col, vals) with vals of shape (4, nnz):
    the input of msgpu_upload_hamiltonian_terms, whose coefficients are then
    (1, Bx, By, Bz).  Each term stores explicit zeros where the others have
    entries, so every field direction shares the pattern."""
    import scipy.sparse as sp
    base = SpinSystem(mult=list(system.mult), names=list(system.names), electrons=system.electrons,
                      bilinear=list(system.bilinear))
    mats = []
    for sysk in [base] + [None] * 3:
        if sysk is None:
            sysk = SpinSystem(mult=list(system.mult), names=list(system.names), electrons=system.electrons)
            _zeeman(sysk, np.eye(3)[len(mats) - 1])
        r, c, v = sysk.hamiltonian_csr()
        D = len(r) - 1
        mats.append(sp.csr_matrix((v, c, r), shape=(D, D)))
    pattern = sum(abs(m) for m in mats).tocsr()
    pattern.sort_indices()
    rows = np.repeat(np.arange(pattern.shape[0]), np.diff(pattern.indptr))
    vals = np.stack([np.asarray(m[rows, pattern.indices]).ravel() for m in mats]).astype(np.complex128)
    return pattern.indptr.astype(np.int32), pattern.indices.astype(np.int32), vals


def _hyperfine(sys_: SpinSystem, e: int, n: int, A_mT: np.ndarray, g: float = G_ELECTRON):
    sys_.bilinear.append((e, n, COMMON_PREFACTOR * 1e-3 * g * np.asarray(A_mT, dtype=np.float64)))


def _random_rotation(rng: np.random.Generator) -> np.ndarray:
    q, r = np.linalg.qr(rng.normal(size=(3, 3)))
    q = q @ np.diag(np.sign(np.diag(r)))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def _aniso_tensor(rng: np.random.Generator, half_range: float) -> np.ndarray:
    ev = rng.uniform(-half_range, half_range, size=3)
    R = _random_rotation(rng)
    return R @ np.diag(ev) @ R.T


def radical_pair(nuc_a: list[int], nuc_b: list[int], couplings_a, couplings_b, field_T,
                 sink_rate: float, st_rate: float = 0.0) -> SpinSystem:
    """Two electrons (leading spins) + nuclei on radical A then B.
    couplings_*: per nucleus either a scalar (isotropic, mT) or a 3x3 tensor (mT)."""
    mult = [2, 2] + list(nuc_a) + list(nuc_b)
    names = ["E1", "E2"] + [f"NA{i}" for i in range(len(nuc_a))] + [f"NB{i}" for i in range(len(nuc_b))]
    s = SpinSystem(mult=mult, names=names, electrons=(0, 1))
    _zeeman(s, field_T)
    for i, a in enumerate(couplings_a):
        _hyperfine(s, 0, 2 + i, np.eye(3) * a if np.isscalar(a) else a)
    for i, a in enumerate(couplings_b):
        _hyperfine(s, 1, 2 + len(nuc_a) + i, np.eye(3) * a if np.isscalar(a) else a)
    s.sinks = {"S": sink_rate, "T0": sink_rate, "Tp": sink_rate, "Tm": sink_rate}
    s.st_rate = st_rate
    return s


@dataclass
class Workload:
    name: str
    system: SpinSystem
    M: int
    dt: float
    steps: int
    krylov: int
    precision: str
    seed: float = 1.0

    @property
    def total_time(self) -> float:
        return self.dt * self.steps

    def times(self) -> np.ndarray:
        return time_grid(self.total_time, self.dt)


def plain_small() -> Workload:
    """2 e (g=2.0023) + 4 I=1/2 on e1, D=64; iso a ~ U[-1,1] mT (seed 0);
    B = 50 uT along z; singlet x 256 SU(Z) samples; k = 1/us; m=16, dt=1 ns, 5000 steps."""
    rng = np.random.default_rng(0)
    a = rng.uniform(-1.0, 1.0, size=4)
    s = radical_pair([2] * 4, [], list(a), [], [0.0, 0.0, 50e-6], sink_rate=1e-3)
    return Workload("plain-small D=64 M=256 m=16 dt=1ns 5000 steps", s, M=256, dt=1.0, steps=5000, krylov=16,
                    precision="c128", seed=1.0)


def precision_large(M: int = 1024, steps: int = 10000) -> Workload:
    """2 e + 12 I=1/2 (8 on A, 4 on B), D=16384; anisotropic symmetric A with
    eigenvalues U[-1.5,1.5] mT, random rotations (seed 1); B = 50 uT random
    direction; 1024 trajectories; m=20, dt=0.5 ns, 10000 steps; complex64 bulk."""
    rng = np.random.default_rng(1)
    ta = [_aniso_tensor(rng, 1.5) for _ in range(8)]
    tb = [_aniso_tensor(rng, 1.5) for _ in range(4)]
    d = rng.normal(size=3)
    d /= np.linalg.norm(d)
    s = radical_pair([2] * 8, [2] * 4, ta, tb, 50e-6 * d, sink_rate=1e-3)
    return Workload("precision-large D=16384 M=1024 m=20 dt=0.5ns 10000 steps", s, M=M, dt=0.5, steps=steps,
                    krylov=20, precision="c64", seed=1.0)


def dense_tc(M: int = 4096, steps: int = 20000) -> Workload:
    """2 e + 8 I=1/2, D=1024, anisotropic (seed 3); dt = 1 ns."""
    rng = np.random.default_rng(3)
    na = 5
    ta = [_aniso_tensor(rng, 1.5) for _ in range(na)]
    tb = [_aniso_tensor(rng, 1.5) for _ in range(8 - na)]
    d = rng.normal(size=3)
    d /= np.linalg.norm(d)
    s = radical_pair([2] * na, [2] * (8 - na), ta, tb, 50e-6 * d, sink_rate=1e-3)
    return Workload("dense D=1024 M=4096 dt=1ns 20000 steps", s, M=M, dt=1.0, steps=steps, krylov=16,
                    precision="c64", seed=3.0)


def batching_systems(n: int = 64, seed: int = 4, steps: int = 4000) -> list[Workload]:
    """64 radical pairs with 4-10 nuclei, 0-2 of them I=1 and the rest I=1/2
    (dims 64..9216), iso a ~ U[-1,1] mT, |B| ~ U[0,1] mT (random direction),
    M ~ U[64,1024], k ~ U[0.5,2]/us, dt=1 ns, 4000 steps, m=16 (reference default)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        ntot = int(rng.integers(4, 11))
        nn = int(rng.integers(0, 3))
        nh = ntot - nn
        nuc = [2] * nh + [3] * nn
        split = int(rng.integers(1, len(nuc) + 1)) if len(nuc) > 1 else len(nuc)
        na, nb = nuc[:split], nuc[split:]
        ca = list(rng.uniform(-1, 1, size=len(na)))
        cb = list(rng.uniform(-1, 1, size=len(nb)))
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        B = rng.uniform(0.0, 1e-3) * d
        k = rng.uniform(0.5e-3, 2e-3)
        s = radical_pair(na, nb, ca, cb, B, sink_rate=k)
        M = int(rng.integers(64, 1025))
        out.append(Workload(f"batch[{i}] D={s.dim} M={M}", s, M=M, dt=1.0, steps=steps, krylov=16,
                            precision="c64", seed=float(i + 1)))
    return out


def serving_request(req_id: int, grid: np.ndarray | None = None, nuclei: tuple[int, int] = (6, 14),
                    steps: int = 3000) -> Workload:
    """One serving request: 6-14 I=1/2 (D=256..65536), anisotropic tensors seeded
    by the request id, one orientation of a 200-point sphere grid at 50 uT,
    256 trajectories, ST dephasing 0.1/us, k = 1/us, 3 us at dt = 1 ns."""
    rng = np.random.default_rng(10_000 + req_id)
    nh = int(rng.integers(nuclei[0], nuclei[1] + 1))
    na = int(rng.integers(1, nh))
    ta = [_aniso_tensor(rng, 1.5) for _ in range(na)]
    tb = [_aniso_tensor(rng, 1.5) for _ in range(nh - na)]
    if grid is None:
        grid = sphere_grid(200)
    d = grid[int(rng.integers(0, len(grid)))]
    s = radical_pair([2] * na, [2] * (nh - na), ta, tb, 50e-6 * d, sink_rate=1e-3, st_rate=1e-4)
    return Workload(f"request {req_id} D={s.dim}", s, M=256, dt=1.0, steps=steps, krylov=16, precision="c64",
                    seed=float(req_id + 1))


def sphere_grid(n: int) -> np.ndarray:
    """Golden-angle sphere points, the "uniform" powder grid of
    SpinAPI/PowderGrid.cpp:144-168 (CreateUniformPowderGrid, full sphere)."""
    k = np.arange(n) + 0.5
    z = 1.0 - 2.0 * k / n
    phi = k * math.pi * (3.0 - math.sqrt(5.0))
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)


def time_grid(total: float, dt: float) -> np.ndarray:
    """Exact-endpoint free-evolution grid (TaskHSGeneral.cpp:59-96)."""
    from . import _lib as L
    n = L.lib.msgpu_host_time_grid(float(total), float(dt), None, 0)
    if n < 0:
        raise ValueError("invalid time grid")
    t = np.zeros(n, dtype=np.float64)
    L.lib.msgpu_host_time_grid(float(total), float(dt), L.dptr(t), n)
    return t
