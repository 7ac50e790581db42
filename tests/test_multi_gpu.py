"""Several right-hand sides of one system (tbs_solve_multi) on the GPU.

The multi-RHS kernels read the line blocks once per sweep for a group of up
to 8 right-hand sides but keep the single-system kernels' per-element
arithmetic and norm order, and retire each right-hand side at the sweep
where a solve of it alone stops.  So every right-hand side's solution,
sweep count and norm history must be bit-identical to set_rhs + solve of
it alone (exact equality), on meshes with ragged lines, single-cell lines,
one-line meshes, groups of 1..8 and more than 8 (several groups), rows that
converge at different sweeps, zero rows and sweep limits.  The alone solves
are pinned to the CPU oracle by test_parity_gpu.py; one multi solve is also
checked against the oracle here.
"""
import numpy as np
import pytest

import oracle
from meshes import ragged_mesh
from triblocksolve_b200 import ALGO_FP64, ALGO_MIXED, Jacobian, Mesh, Solver
from triblocksolve_b200._native import TbsError

pytestmark = pytest.mark.gpu

SYSTEMS = [
    (lambda: Mesh.structured(24, 40), 9.0, 1),
    (lambda: ragged_mesh([5, 1, 7, 3, 3, 8, 13, 2, 9], seed=4), 9.0, 2),
    (lambda: Mesh.structured(1, 37), 9.0, 3),
    (lambda: Mesh.structured(6, 1), 9.0, 4),
    (lambda: Mesh.structured(7, 11), 4.0, 5),
    (lambda: Mesh.structured(1, 1), 9.0, 6),
    (lambda: Mesh.structured(40, 96), 6.0, 7),
]
TOL = 1e-11


def solver_for(mesh, jac):
    s = Solver(0)
    s.set_mesh(mesh)
    s.set_jacobian(jac)
    s.factor(ALGO_FP64)
    return s


def rows_for(mesh, nrhs, seed):
    """Right-hand sides that converge at different sweeps: random rows,
    smooth rows, a row concentrated on a few cells, and a zero row."""
    rng = np.random.default_rng(seed)
    n = 9 * mesh.nelem
    out = []
    for k in range(nrhs):
        kind = k % 4
        if kind == 0:
            out.append(rng.uniform(-1, 1, n))
        elif kind == 1:
            x = np.linspace(0, 1, n)
            out.append(np.sin(3 * np.pi * x + k) * (1 + k))
        elif kind == 2:
            v = np.zeros(n)
            v[rng.integers(0, n, size=max(1, n // 50))] = rng.uniform(-5, 5, max(1, n // 50))
            out.append(v)
        else:
            out.append(np.zeros(n) if k == 3 else rng.uniform(-1e-3, 1e-3, n))
    return np.array(out)


def check_vs_alone(s, rhs, U, sw, hist, tol, max_sweeps):
    for r in range(rhs.shape[0]):
        s.set_rhs(rhs[r])
        n1, h1 = s.solve(tol, max_sweeps)
        assert sw[r] == n1, (r, sw[r], n1)
        np.testing.assert_array_equal(hist[r], h1)
        np.testing.assert_array_equal(U[r], s.solution())


@pytest.mark.parametrize("k", range(len(SYSTEMS)))
@pytest.mark.parametrize("nrhs", [1, 3, 8])
def test_multi_equals_alone(k, nrhs):
    mk, shift, seed = SYSTEMS[k]
    mesh = mk()
    jac = Jacobian.generate(mesh, shift, seed)
    s = solver_for(mesh, jac)
    try:
        rhs = rows_for(mesh, nrhs, 10 * k + nrhs)
        U, sw, hist = s.solve_multi(rhs, TOL, 200)
        check_vs_alone(s, rhs, U, sw, hist, TOL, 200)
    finally:
        s.close()


def test_several_groups_and_limits():
    mesh = Mesh.structured(40, 96)
    jac = Jacobian.generate(mesh, 4.0, 11)
    s = solver_for(mesh, jac)
    try:
        rhs = rows_for(mesh, 19, 5)  # groups of 8, 8, 3
        # rows whose error is already smooth (the residual after k sweeps of
        # another row) need more sweeps to reach the relative tolerance
        for j, k in enumerate((2, 4, 6)):
            s.set_rhs(rhs[j])
            s.sweep(k)
            rhs[4 + j] = s.residual()
        U, sw, hist = s.solve_multi(rhs, TOL, 200)
        assert len(set(sw[:8].tolist())) > 2  # rows of one group retire at different sweeps
        check_vs_alone(s, rhs, U, sw, hist, TOL, 200)
        # a sweep limit that stops some rows before their tolerance
        U, sw, hist = s.solve_multi(rhs[:8], TOL, 3)
        assert sw.max() == 3
        check_vs_alone(s, rhs[:8], U, sw, hist, TOL, 3)
        # zero sweeps allowed
        U, sw, hist = s.solve_multi(rhs[:2], TOL, 0)
        assert not sw.any() and not U.any()
    finally:
        s.close()


def test_multi_matches_oracle():
    mesh = Mesh.structured(12, 16)
    jac = Jacobian.generate(mesh, 9.0, 3)
    s = solver_for(mesh, jac)
    try:
        rhs = rows_for(mesh, 3, 1)[:3]
        U, sw, hist = s.solve_multi(rhs, 0.0, 12)
        assert (sw == 12).all()
        for r in range(3):
            ref = oracle.lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, rhs[r], 12)
            # FP64 form vs the reference operation order: every sweep's norm
            # within 1e-12 ||R_0||, U within 1e-12 ||U||
            np.testing.assert_allclose(hist[r], ref["hist"], rtol=0, atol=1e-12 * ref["hist"][0])
            assert np.linalg.norm(U[r] - ref["U"]) <= 1e-12 * np.linalg.norm(ref["U"])
    finally:
        s.close()


def test_device_buffers_and_context_untouched():
    import torch

    mesh = Mesh.structured(24, 40)
    jac = Jacobian.generate(mesh, 9.0, 1)
    s = solver_for(mesh, jac)
    try:
        n0, h0 = s.solve(TOL, 200)
        U0 = s.solution()
        rhs = rows_for(mesh, 5, 2)
        d_rhs = torch.from_numpy(rhs).cuda()
        d_U = torch.zeros_like(d_rhs)
        torch.cuda.synchronize()  # the context works on its own stream
        sw, hist = s.solve_multi_device(d_rhs.data_ptr(), d_U.data_ptr(), 5, TOL, 200)
        U = d_U.cpu().numpy()
        # the context's own solve is not disturbed
        np.testing.assert_array_equal(s.solution(), U0)
        check_vs_alone(s, rhs, U, sw, hist, TOL, 200)
    finally:
        s.close()


def test_multi_errors():
    mesh = Mesh.structured(6, 8)
    jac = Jacobian.generate(mesh, 9.0, 1)
    s = Solver(0)
    try:
        s.set_mesh(mesh)
        s.set_jacobian(jac)
        with pytest.raises(TbsError):
            s.solve_multi(np.zeros((2, 9 * mesh.nelem)), TOL, 10)  # not factored
        s.factor(ALGO_MIXED)
        with pytest.raises(TbsError):
            s.solve_multi(np.zeros((2, 9 * mesh.nelem)), TOL, 10)  # FP64 only
        s.factor(ALGO_FP64)
        with pytest.raises(TbsError):
            s.solve_multi(np.zeros((2, 9 * mesh.nelem)), -1.0, 10)
    finally:
        s.close()


def test_results_into_caller_arrays():
    """solution(out=...) and solve_multi(out=...) fill the caller's (pinned)
    arrays with exactly what the allocating forms return; wrong shapes are
    refused before any copy."""
    import torch
    mesh = Mesh.structured(10, 12)
    jac = Jacobian.generate(mesh, 9.0, 5)
    s = Solver(0)
    s.set_mesh(mesh)
    s.set_jacobian(jac)
    s.factor(ALGO_FP64)
    s.solve(1e-12, 100)
    n = 9 * mesh.nelem
    pinned = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    assert s.solution(out=pinned) is pinned
    assert np.array_equal(pinned, s.solution())
    with pytest.raises(ValueError):
        s.solution(out=np.zeros(n - 1))
    rows = np.stack([jac.rhs, -jac.rhs])
    U, sw, _h = s.solve_multi(rows, 1e-12, 100)
    out = torch.empty((2, n), dtype=torch.float64, pin_memory=True).numpy()
    U2, sw2, _h2 = s.solve_multi(rows, 1e-12, 100, out=out)
    assert np.array_equal(out, U) and np.array_equal(sw, sw2)
    s.close()
