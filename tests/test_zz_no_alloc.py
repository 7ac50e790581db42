"""tbs_residual_noalloc: the residual entry point for callers that cannot
allocate device memory (a solver whose pool owns the GPU, a time loop that
must not allocate).  It keeps its work array in a fixed device array instead
of cudaMalloc; here it is checked, on two calls in a row, against the
context API's residual (tbs_get_residual / tbs_true_residual_norm) and the
oracle's (the reference's residual rule restated on the CPU) with the
parity tolerance of the other GPU tests (1e-12 of the initial residual),
on the legacy default stream and on a stream of the caller's.
This file sorts last so that a run stopping at the first failure has already
run every other test."""
import ctypes as C

import numpy as np
import pytest

import oracle
from meshes import ragged_mesh
from triblocksolve_b200 import ALGO_FP64, ALGO_REFERENCE, Jacobian, Mesh, Solver
from triblocksolve_b200 import _native as N

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _noalloc(mesh, bufs, U, want_R=True, stream=None):
    import torch
    dU = _dev(U)
    dR = torch.empty_like(dU) if want_R else None
    norm = C.c_double(-1.0)
    torch.cuda.synchronize()
    rc = N.lib.tbs_residual_noalloc(0, stream, mesh.nelem, bufs["epoint"].data_ptr(),
                                    bufs["ef"].data_ptr(), bufs["fc"].data_ptr(),
                                    bufs["jacD"].data_ptr(), bufs["jacO1"].data_ptr(),
                                    bufs["jacO2"].data_ptr(), bufs["rhs"].data_ptr(),
                                    dU.data_ptr(), dR.data_ptr() if want_R else None,
                                    C.byref(norm))
    N.check(rc)
    return (dR.cpu().numpy() if want_R else None), norm.value


@pytest.mark.parametrize("algo", [ALGO_FP64, ALGO_REFERENCE])
@pytest.mark.parametrize("make", [lambda: Mesh.structured(60, 64),
                                  lambda: ragged_mesh([5, 1, 7, 3, 3, 8, 13, 2, 9], seed=4)])
def test_noalloc_residual_matches_context(algo, make):
    mesh = make()
    jac = Jacobian.generate(mesh, 9.0, 3)
    s = Solver(0)
    s.set_mesh(mesh)
    s.set_jacobian(jac)
    s.factor(algo)
    bufs = {f: _dev(getattr(mesh, f)) for f in ("epoint", "ef", "fc")}
    bufs.update({f: _dev(getattr(jac, f)) for f in ("jacD", "jacO1", "jacO2", "rhs")})
    tol = 1e-12 * np.linalg.norm(jac.rhs)
    for sweeps in (2, 3):  # two calls in a row on different iterates
        s.sweep(sweeps)
        U = s.solution()
        R_ctx = s.residual()
        n_ctx = s.true_residual_norm()
        R, nrm = _noalloc(mesh, bufs, U)
        assert np.max(np.abs(R - R_ctx)) <= tol
        assert abs(nrm - n_ctx) <= tol
        assert abs(nrm - np.linalg.norm(R)) <= tol
    _, nrm = _noalloc(mesh, bufs, s.solution(), want_R=False)
    assert abs(nrm - s.true_residual_norm()) <= tol
    s.close()


def test_noalloc_on_a_caller_stream_matches_oracle():
    """The call on a stream of the caller's (ticket clear, kernel, norm copy
    and synchronisation all on it), two calls in a row, against the oracle's
    residual (the reference's lineRes rule restated on the CPU) and the
    context path."""
    import torch
    mesh = ragged_mesh([12, 3, 9, 16, 1, 7], seed=6)
    jac = Jacobian.generate(mesh, 9.0, 5)
    bufs = {f: _dev(getattr(mesh, f)) for f in ("epoint", "ef", "fc")}
    bufs.update({f: _dev(getattr(jac, f)) for f in ("jacD", "jacO1", "jacO2", "rhs")})
    s = Solver(0)
    s.set_mesh(mesh)
    s.set_jacobian(jac)
    s.factor(ALGO_FP64)
    st = torch.cuda.Stream()
    tol = 1e-12 * np.linalg.norm(jac.rhs)
    for sweeps in (1, 2):
        s.sweep(sweeps)
        U = s.solution()
        R, nrm = _noalloc(mesh, bufs, U, stream=C.c_void_p(st.cuda_stream))
        R_or = oracle.true_residual(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, U)
        assert np.max(np.abs(R - R_or)) <= tol
        assert abs(nrm - np.linalg.norm(R_or)) <= tol
        assert abs(nrm - s.true_residual_norm()) <= tol
    s.close()


def test_noalloc_rejects_oversize_and_nulls():
    dummy = C.c_void_p(1)
    norm = C.c_double()
    rc = N.lib.tbs_residual_noalloc(0, None, 2_097_153, dummy, dummy, dummy, dummy, dummy, dummy,
                                    dummy, dummy, None, C.byref(norm))
    assert rc == N.TBS_ERR_ARG and "limit" in N.last_error()
    rc = N.lib.tbs_residual_noalloc(0, None, 10, None, dummy, dummy, dummy, dummy, dummy, dummy,
                                    dummy, None, C.byref(norm))
    assert rc == N.TBS_ERR_ARG
