"""The allocation-free Krylov step (msgpu_krylov_step_noalloc).

Callers that cannot allocate device memory -- hosts whose memory pool owns
every allocation, code that must not take the implicit device
synchronisation of cudaMalloc / cudaFree -- get one Krylov step that
uses only their buffers and the library's static scratch area.  Here it is
called through the C ABI with caller-owned device buffers and compared with
the regular entry point (msgpu_run of one step followed by
msgpu_download_factors) on two calls in a row, the second starting from the
first one's output so that stale scratch contents would show up.  The file
name sorts last so that a stop-at-first-failure run has already run every
other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _one_step_with_run(system, psi, dt, m):
    from molspin_b200 import hsgeneral as hs
    with hs.HSPropagatorB200(0) as p:
        p.set_hamiltonian(*system.hamiltonian_csr())
        p.set_reaction(kappa=system.kappa())
        p.set_electron_pair(*system.electron_strides())
        p.set_observables([(op, rate) for _, op, rate in system.observables()])
        p.set_factors(psi)
        p.propagate(np.array([0.0, dt]), m, "c128")
        return p.get_factors()


def test_noalloc_step_matches_regular_entry_point_twice():
    import torch

    from molspin_b200 import _lib as L
    from molspin_b200 import systems as S

    system = S.plain_small().system
    D, M, dt, m = system.dim, 96, 1.0, 16
    r, c, v = system.hamiltonian_csr()
    kappa = system.kappa()
    dev = torch.device("cuda", 0)
    # caller-owned device buffers (allocated here by the caller, not by the library)
    d_row = torch.from_numpy(np.ascontiguousarray(r)).to(dev)
    d_col = torch.from_numpy(np.ascontiguousarray(c)).to(dev)
    d_val = torch.from_numpy(np.ascontiguousarray(v).view(np.float64)).to(dev)
    stream = torch.cuda.current_stream(dev)
    psi = system.trace_samples(M, 1.0)
    for call in range(2):
        ref = _one_step_with_run(system, psi, dt, m)
        d_in = torch.from_numpy(np.ascontiguousarray(psi.T).view(np.float64).copy()).to(dev)
        d_out = torch.full_like(d_in, float("nan"))
        torch.cuda.synchronize()
        rc = L.lib.msgpu_krylov_step_noalloc(D, d_row.data_ptr(), d_col.data_ptr(), d_val.data_ptr(), kappa, M,
                                             d_in.data_ptr(), d_out.data_ptr(), dt, m, stream.cuda_stream)
        assert rc == L.MSGPU_OK, f"call {call}: rc={rc}"
        got = d_out.cpu().numpy().view(np.complex128).reshape(M, D).T
        err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
        assert err < 1e-12, f"call {call}: relative deviation {err:.3e}"
        psi = got

    # problems larger than the static scratch area are refused before any
    # work, the largest trajectory count included (no index overflow)
    for big in (1 << 16, 2 ** 31 - 1):
        rc = L.lib.msgpu_krylov_step_noalloc(D, d_row.data_ptr(), d_col.data_ptr(), d_val.data_ptr(), kappa, big,
                                             d_in.data_ptr(), d_out.data_ptr(), dt, m, stream.cuda_stream)
        assert rc == L.MSGPU_ERR_SCRATCH, (big, rc)
