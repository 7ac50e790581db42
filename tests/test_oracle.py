"""The CPU oracle: pinned to the committed fixture, to an independent dense
numpy statement of the LIJ iteration, and to the library's host helpers."""
import json
import os

import numpy as np
import pytest

import oracle
from meshes import ragged_mesh
from triblocksolve_b200 import Jacobian, Mesh

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def blocks(arr, nv):
    """column-major (i + nv*j + nv*nv*b) -> [b, i, j]"""
    return arr.reshape(-1, nv, nv).transpose(0, 2, 1)


def dense_system(mesh, jac):
    nv, ne = mesh.nvar, mesh.nelem
    D, O1, O2 = blocks(jac.jacD, nv), blocks(jac.jacO1, nv), blocks(jac.jacO2, nv)
    J = np.zeros((nv * ne, nv * ne))
    M = np.zeros_like(J)

    def put(A, r, c, B):
        A[nv * r:nv * r + nv, nv * c:nv * c + nv] += B

    for e in range(ne):
        put(J, e, e, D[e])
        put(M, e, e, D[e])
        for k2 in range(mesh.epoint[e], mesh.epoint[e + 1]):
            f = mesh.ef[k2]
            if f < 0:
                continue
            e1, e2 = mesh.fc[2 * f], mesh.fc[2 * f + 1]
            if e == e1:
                put(J, e, e2, O2[f])
            else:
                put(J, e, e1, O1[f])
    for l in range(mesh.nline):
        for k in range(1, mesh.linesize[l]):
            m = mesh.linepoint[l] + k
            f = mesh.lineface[m]
            e, ep = mesh.lines[m], mesh.lines[m - 1]
            e1 = mesh.fc[2 * f]
            put(M, e, ep, O2[f] if e == e1 else O1[f])
            put(M, ep, e, O1[f] if e == e1 else O2[f])
    return J, M


def dense_lij(mesh, jac, iters):
    J, M = dense_system(mesh, jac)
    U = np.zeros(J.shape[0])
    R = jac.rhs.copy()
    hist = [np.linalg.norm(R)]
    for _ in range(iters):
        dU = -np.linalg.solve(M, R)
        U = U + dU
        R = jac.rhs + J @ U
        hist.append(np.linalg.norm(R))
    return U, R, np.array(hist)


def test_oracle_matches_committed_fixture():
    g = json.load(open(os.path.join(GOLD, "lij_60x64.json")))
    p = g["problem"]
    m = Mesh.structured(p["L"], p["K"])
    j = Jacobian.generate(m, p["shift"], p["seed"])
    r = oracle.lij(m, j.jacD, j.jacO1, j.jacO2, j.rhs, p["sweeps"], threads=1)
    # the fixture is the reference's own kernels' output: equal bit for bit
    np.testing.assert_array_equal(r["hist"], g["hist"])
    assert float(r["U"].sum()) == g["U_sum"] and float((r["U"] * r["U"]).sum()) == g["U_sumsq"]
    np.testing.assert_array_equal(r["U"][:9], g["U_first"])
    np.testing.assert_array_equal(r["U"][-9:], g["U_last"])


@pytest.mark.parametrize("lens,shift,seed", [([6, 6, 6, 6], 9.0, 1), ([5, 1, 7, 3, 3, 8], 4.0, 2),
                                             ([1, 1, 1], 9.0, 3), ([12], 9.0, 4)])
def test_oracle_against_dense_lij(lens, shift, seed):
    m = ragged_mesh(lens, seed=seed)
    j = Jacobian.generate(m, shift, seed)
    U_ref, R_ref, hist_ref = dense_lij(m, j, 8)
    r = oracle.lij(m, j.jacD, j.jacO1, j.jacO2, j.rhs, 8)
    scale = np.linalg.norm(U_ref)
    assert np.linalg.norm(r["U"] - U_ref) <= 1e-12 * scale
    np.testing.assert_allclose(r["hist"], hist_ref, rtol=0, atol=1e-12 * hist_ref[0])
    np.testing.assert_allclose(r["R"], R_ref, rtol=0, atol=1e-12 * hist_ref[0])


def test_oracle_is_thread_count_independent():
    m = Mesh.structured(20, 30)
    j = Jacobian.generate(m, 9.0, 5)
    a = oracle.lij(m, j.jacD, j.jacO1, j.jacO2, j.rhs, 5, threads=1)
    b = oracle.lij(m, j.jacD, j.jacO1, j.jacO2, j.rhs, 5, threads=4)
    for k in ("U", "R", "dU", "hist"):
        np.testing.assert_array_equal(a[k], b[k])


def test_oracle_converges_and_detects_tolerance():
    m = Mesh.structured(12, 16)
    j = Jacobian.generate(m, 4.0, 9)
    r = oracle.lij(m, j.jacD, j.jacO1, j.jacO2, j.rhs, 15)
    rel = r["hist"] / r["hist"][0]
    assert rel[-1] < 1e-10
    assert np.all(np.diff(rel[:8]) < 0)
    R = oracle.true_residual(m, j.jacD, j.jacO1, j.jacO2, j.rhs, r["U"])
    np.testing.assert_array_equal(R, r["R"])


@pytest.mark.parametrize("nv_new", [12, 5, 9])
def test_resize_block_size_matches_oracle(nv_new):
    m = Mesh.structured(3, 4)
    j = Jacobian.generate(m, 9.0, 2)
    want = oracle.resize_block_size(9, nv_new, m.nelem, m.nintface, j.jacD, j.jacO1, j.jacO2,
                                    j.rhs, j.U0)
    j.resizeBlockSize(nv_new)
    for a, b in zip((j.jacD, j.jacO1, j.jacO2, j.rhs, j.U0), want):
        np.testing.assert_array_equal(a, b)
    assert j.nvar == nv_new


def test_assemble_triblocks_matches_oracle():
    import ctypes as C
    m = ragged_mesh([5, 2, 6, 4], seed=8)
    j = Jacobian.generate(m, 9.0, 8)
    j.assembleTriBlocks(m)
    A = np.zeros(81 * m.nelem)
    keep = [np.ascontiguousarray(getattr(m, f), np.int32) for f in
            ("fc", "linesize", "linepoint", "lines", "lineface")]
    ip = C.POINTER(C.c_int)
    dp = C.POINTER(C.c_double)
    oracle.lib.oracle_assemble_A(9, m.nline, *[a.ctypes.data_as(ip) for a in keep],
                                 j.jacO1.ctypes.data_as(dp), j.jacO2.ctypes.data_as(dp),
                                 A.ctypes.data_as(dp))
    np.testing.assert_array_equal(j.A[:A.size], A)


@pytest.mark.parametrize("lens,shift,seed", [([6, 6, 6, 6], 9.0, 1), ([5, 1, 7, 3, 3, 8], 4.0, 2),
                                             ([12], 9.0, 4)])
def test_oracle_pij_against_dense(lens, shift, seed):
    """oracle.pij (the line sweep on one-cell lines) is the point-implicit
    Jacobi iteration dU = -D^-1 R, U += dU, R = rhs + J U, written densely."""
    m = ragged_mesh(lens, seed=seed)
    j = Jacobian.generate(m, shift, seed)
    J, _ = dense_system(m, j)
    nv = m.nvar
    D = blocks(j.jacD, nv)
    U = np.zeros(J.shape[0])
    R = j.rhs.copy()
    hist = [np.linalg.norm(R)]
    for _ in range(8):
        dU = -np.linalg.solve(D, R.reshape(-1, nv, 1)).reshape(-1)
        U = U + dU
        R = j.rhs + J @ U
        hist.append(np.linalg.norm(R))
    r = oracle.pij(m, j.jacD, j.jacO1, j.jacO2, j.rhs, 8)
    assert np.linalg.norm(r["U"] - U) <= 1e-12 * np.linalg.norm(U)
    np.testing.assert_allclose(r["hist"], hist, rtol=0, atol=1e-12 * hist[0])
    # it converges more slowly than the line sweep on the same system
    lij = oracle.lij(m, j.jacD, j.jacO1, j.jacO2, j.rhs, 8)
    if len(lens) > 1:
        assert lij["hist"][-1] < r["hist"][-1]


@pytest.mark.parametrize("restart,psweeps", [(30, 1), (4, 1), (6, 2)])
def test_oracle_gmres_solves_the_dense_system(restart, psweeps):
    """oracle.gmres (line-preconditioned GMRES over the oracle's own sweep
    and residual) reaches the solution of the dense system J U = -rhs."""
    m = ragged_mesh([5, 1, 7, 3, 3, 8], seed=2)
    j = Jacobian.generate(m, 2.5, 2)  # weak diagonal: plain line sweeps are slow here
    J, _ = dense_system(m, j)
    U_exact = np.linalg.solve(J, -j.rhs)
    r = oracle.gmres(m, j.jacD, j.jacO1, j.jacO2, j.rhs, restart, psweeps, 1e-11, 200)
    assert r["hist"][-1] <= 1e-11 * r["hist"][0]
    assert np.linalg.norm(r["U"] - U_exact) <= 1e-9 * np.linalg.norm(U_exact)
    # far fewer preconditioner applications than plain line sweeps to 1e-11
    lij = oracle.lij(m, j.jacD, j.jacO1, j.jacO2, j.rhs, 200)
    n_lij = int(np.argmax(lij["hist"] <= 1e-11 * lij["hist"][0]))
    assert 2 * r["iters"] * psweeps < n_lij
