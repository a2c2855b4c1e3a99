"""Exact density-matrix FP64 oracle for small systems (numpy/scipy).

TEST INFRASTRUCTURE ONLY.  Builds H by dense Kronecker products of the spin
matrices (independently of the product's CSR assembly) and propagates
rho = E[|psi><psi|] with the same symmetric split the stochastic path samples:

    rho <- R(h) rho ;  rho <- E rho E^+ ;  rho <- R(h) rho,
    E = exp(dt G), G = -iH - K, R(h) rho = (1-p) rho + p U rho U^+,
    p = -expm1(-2 lambda h)/2, lambda = k_ST/2, U = PS - PT,

exactly the density recursion of the reference's SplitConvergence and
NoncommutingMonteCarloConvergence tests (Tests/tests_StochasticRelaxation.cpp:
371-397, 466-499).  Observables are rate * Tr(O rho) and the yields their
trapezoid integrals on the same grid (HSObservableCollector.cpp:304-326).
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp


def spin_matrices(mult: int):
    S = 0.5 * (mult - 1)
    m = S - np.arange(mult)
    Sz = np.diag(m).astype(np.complex128)
    Sp = np.zeros((mult, mult), dtype=np.complex128)
    for i in range(mult - 1):
        Sp[i, i + 1] = np.sqrt(S * (S + 1) - m[i] * (m[i] - 1))
    Sx = 0.5 * (Sp + Sp.T)
    Sy = -0.5j * (Sp - Sp.T)
    return Sx, Sy, Sz


def embed(ops: dict[int, np.ndarray], mult: list[int]) -> np.ndarray:
    out = np.ones((1, 1), dtype=np.complex128)
    for k, d in enumerate(mult):
        out = np.kron(out, ops.get(k, np.eye(d)))
    return out


def dense_hamiltonian(system) -> np.ndarray:
    mult = system.mult
    D = int(np.prod(mult))
    H = np.zeros((D, D), dtype=np.complex128)
    S = [spin_matrices(d) for d in mult]
    for k, w in system.linear:
        for a in range(3):
            if w[a] != 0.0:
                H += w[a] * embed({k: S[k][a]}, mult)
    for i, j, Cm in system.bilinear:
        for a in range(3):
            for b in range(3):
                if Cm[a][b] != 0.0:
                    H += Cm[a][b] * embed({i: S[i][a]}, mult) @ embed({j: S[j][b]}, mult)
    return H


def _sparse_embed(ops: dict, mult: list[int]):
    out = sp.identity(1, dtype=np.complex128, format="csr")
    for k, d in enumerate(mult):
        out = sp.kron(out, sp.csr_matrix(ops[k]) if k in ops else sp.identity(d, dtype=np.complex128), format="csr")
    return out


def sparse_hamiltonian(system):
    """H as CSR (rowptr, col, val) for dimensions where the dense assembly does not fit: the same
    Kronecker terms as dense_hamiltonian, with scipy.sparse products."""
    mult = system.mult
    S = [spin_matrices(d) for d in mult]
    D = int(np.prod(mult))
    H = sp.csr_matrix((D, D), dtype=np.complex128)
    for k, w in system.linear:
        for a in range(3):
            if w[a] != 0.0:
                H = H + w[a] * _sparse_embed({k: S[k][a]}, mult)
    for i, j, Cm in system.bilinear:
        for a in range(3):
            for b in range(3):
                if Cm[a][b] != 0.0:
                    H = H + Cm[a][b] * _sparse_embed({i: S[i][a], j: S[j][b]} if i != j else
                                                     {i: S[i][a] @ S[j][b]}, mult)
    H = H.tocsr()
    H.eliminate_zeros()
    H.sort_indices()
    return (H.indptr.astype(np.int32), H.indices.astype(np.int32), H.data.astype(np.complex128))


def pair_operator_csr(op4: np.ndarray, system):
    """pair_operator as CSR, without forming the dense D x D matrix."""
    e1, e2 = system.electrons
    D = system.dim
    strides = system.strides()
    idx = np.arange(D)
    d1 = (idx // strides[e1]) % 2
    d2 = (idx // strides[e2]) % 2
    base = idx - d1 * strides[e1] - d2 * strides[e2]
    rows, cols, vals = [], [], []
    for a in range(4):
        for b in range(4):
            v = op4[a, b]
            if v == 0:
                continue
            r = np.nonzero((2 * d1 + d2) == a)[0]
            rows.append(r)
            cols.append(base[r] + (b >> 1) * strides[e1] + (b & 1) * strides[e2])
            vals.append(np.full(len(r), v, dtype=np.complex128))
    m = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(D, D))
    m.sum_duplicates()
    m.sort_indices()
    return (m.indptr.astype(np.int32), m.indices.astype(np.int32), m.data.astype(np.complex128))


def pair_operator(op4: np.ndarray, system) -> np.ndarray:
    """Embed a 4x4 operator on the radical pair (basis |e1 e2>, digit 0 = up)."""
    mult = system.mult
    e1, e2 = system.electrons
    D = int(np.prod(mult))
    strides = system.strides()
    out = np.zeros((D, D), dtype=np.complex128)
    idx = np.arange(D)
    d1 = (idx // strides[e1]) % 2
    d2 = (idx // strides[e2]) % 2
    base = idx - d1 * strides[e1] - d2 * strides[e2]
    for a in range(4):
        for b in range(4):
            v = op4[a, b]
            if v == 0:
                continue
            rows = np.nonzero((2 * d1 + d2) == a)[0]
            cols = base[rows] + (b >> 1) * strides[e1] + (b & 1) * strides[e2]
            out[rows, cols] += v
    return out


def st_unitary(system) -> np.ndarray:
    """U = PS - PT = -1/2 I - 2 S1.S2 on the radical pair."""
    e1, e2 = system.electrons
    S1 = spin_matrices(2)
    D = system.dim
    U = -0.5 * np.eye(D, dtype=np.complex128)
    for a in range(3):
        U += -2.0 * embed({e1: S1[a]}, system.mult) @ embed({e2: S1[a]}, system.mult)
    return U


def to_csr(A: np.ndarray, tol: float = 0.0):
    A = np.where(np.abs(A) > tol, A, 0.0)
    m = sp.csr_matrix(A)
    m.sort_indices()
    return (m.indptr.astype(np.int32), m.indices.astype(np.int32), m.data.astype(np.complex128))


# |S> = (|ud> - |du>)/sqrt(2) in the pair basis uu, ud, du, dd (digit 0 = m=+1/2)
SINGLET = np.array([0.0, 1.0, -1.0, 0.0], dtype=np.complex128) / np.sqrt(2.0)


def singlet_density(system) -> np.ndarray:
    """rho0 = |S><S| x I_Z / Z (the trace-sampled initial state's expectation)."""
    P = pair_operator(np.outer(SINGLET, SINGLET.conj()), system)
    return P / np.trace(P).real


def lindblad_exact(H: np.ndarray, K: np.ndarray, rho0: np.ndarray, t: float, U: np.ndarray | None = None,
                   st_rate: float = 0.0) -> np.ndarray:
    """rho(t) of d rho/dt = -i[H,rho] - {K,rho} + lambda (U rho U^+ - rho), lambda = k_ST/2
    (the reference's relaxation superoperator, Tests/tests_StochasticRelaxation.cpp:55-63),
    by the matrix exponential of the row-major vectorised generator."""
    D = H.shape[0]
    I = np.eye(D)
    Lg = -1j * (np.kron(H, I) - np.kron(I, H.T)) - (np.kron(K, I) + np.kron(I, K.T))
    if U is not None and st_rate > 0.0:
        lam = 0.5 * st_rate
        Lg = Lg + lam * (np.kron(U, U.conj()) - np.eye(D * D))
    v = sla.expm(t * Lg) @ rho0.reshape(-1)
    return v.reshape(D, D)


def st_dephasing_rk4(H: np.ndarray, K: np.ndarray, rho0: np.ndarray, times: np.ndarray, observables,
                     U: np.ndarray, st_rate: float) -> np.ndarray:
    """The reference's deterministic ("direct") HSGeneral arm with an ST-dephasing Operator:
    one classical RK4 step of the density matrix per grid interval
    (HSPropagator::StepDensity, RunSection/General/HS/HSPropagator.cpp:152-189) on
        d rho/dt = -i[H, rho] - {K, rho} - k (P_T rho P_S + P_S rho P_T),
    the dephasing term of SpinSpace::ApplyRelaxationHilbert
    (SpinAPI/SpinSpace/SpinSpace_relaxation.cpp:695-716), with P_S = (1 + U)/2,
    P_T = 1 - P_S.  Observables are evaluated before every step
    (TaskHSGeneral.cpp:471-560).  Returns values[(ntimes) x nobs] of rate * Tr(O rho)."""
    D = H.shape[0]
    PS = 0.5 * (np.eye(D) + U)
    PT = np.eye(D) - PS

    def rhs(r):
        return -1j * (H @ r - r @ H) - (K @ r + r @ K) - st_rate * (PT @ r @ PS + PS @ r @ PT)

    rho = rho0.astype(np.complex128).copy()
    values = np.zeros((len(times), len(observables)))
    for s in range(len(times)):
        values[s] = [rate * np.trace(O @ rho).real for O, rate in observables]
        if s + 1 == len(times):
            break
        dt = times[s + 1] - times[s]
        k1 = rhs(rho)
        k2 = rhs(rho + 0.5 * dt * k1)
        k3 = rhs(rho + 0.5 * dt * k2)
        k4 = rhs(rho + dt * k3)
        rho = rho + (dt / 6.0) * (k1 + 2.0 * k2 + 2.0 * k3 + k4)
    return values


def data_file_difference(a: np.ndarray, b: np.ndarray) -> float:
    """max |a - b| over the values as the reference's data file prints them (12 significant
    digits, TaskHSGeneral.cpp:642-646), as Tests/StochasticRelaxation/check_output.py reads them."""
    def printed(x):
        return np.array([[float(f"{v:.12g}") for v in row] for row in np.atleast_2d(x)])
    return float(np.max(np.abs(printed(a) - printed(b))))


def propagate_density(H: np.ndarray, K: np.ndarray, rho0: np.ndarray, times: np.ndarray, observables,
                      U: np.ndarray | None = None, st_rate: float = 0.0, return_rho: bool = False):
    """observables: list of (dense O, rate).  Returns (values[(ntimes) x nobs], yields[nobs])
    (and the final rho when return_rho)."""
    G = -1j * H - K
    rho = rho0.copy()
    nobs = len(observables)
    values = np.zeros((len(times), nobs))
    cache = {}
    lam = 0.5 * st_rate

    def R(rho, h):
        if U is None or lam <= 0.0 or h == 0.0:
            return rho
        p = -0.5 * np.expm1(-2.0 * lam * h)
        return (1 - p) * rho + p * (U @ rho @ U.conj().T)

    for s in range(len(times)):
        values[s] = [rate * np.trace(O @ rho).real for O, rate in observables]
        if s + 1 == len(times):
            break
        dt = times[s + 1] - times[s]
        key = round(dt, 15)
        if key not in cache:
            cache[key] = sla.expm(dt * G)
        E = cache[key]
        rho = R(rho, 0.5 * dt)
        rho = E @ rho @ E.conj().T
        rho = R(rho, 0.5 * dt)
    dts = np.diff(times)
    yields = (0.5 * dts[:, None] * (values[:-1] + values[1:])).sum(axis=0)
    if return_rho:
        return values, yields, rho
    return values, yields


def orthonormal_nuclear_samples(system, state: np.ndarray) -> np.ndarray:
    """M = Z "samples" |pair> x e_j / sqrt(Z): an exact trace estimator."""
    Z = system.dim // 4
    F = np.zeros((system.dim, Z), dtype=np.complex128)
    for j in range(Z):
        e = np.zeros(Z)
        e[j] = 1.0
        F[:, j] = np.kron(state, e) / np.sqrt(Z)
    return F
