"""Line-preconditioned GMRES (tbs_gmres) on the GPU.

The oracle is oracle.gmres: the same restarted GMRES (classical
Gram-Schmidt twice, Givens rotations, true residual at every restart) over
the reference's own sweep loop as preconditioner and its residual rule as
the product with J, pinned to the dense solution by tests/test_oracle.py.
The GPU preconditioner is the TBS_ALGO_FP64 sweep (within 1e-12 of the
reference order per sweep) and its sums run in another order, so the
stated tolerance is: same number of Arnoldi steps, every history entry
within 1e-9 ||rhs||, the solution within 1e-9 (relative), and the true
residual at the requested tolerance.
"""
import numpy as np
import pytest

import oracle
from meshes import ragged_mesh
from triblocksolve_b200 import ALGO_FP64, ALGO_MIXED, Jacobian, Mesh, Solver
from triblocksolve_b200._native import TbsError

pytestmark = pytest.mark.gpu


@pytest.fixture
def solver():
    s = Solver(0)
    yield s
    s.close()


def setup(s, mesh, jac, algo=ALGO_FP64):
    s.set_mesh(mesh)
    s.set_jacobian(jac)
    s.factor(algo)


CASES = [
    ("structured", lambda: Mesh.structured(12, 16), 2.5, 30, 1),
    ("ragged", lambda: ragged_mesh([5, 1, 7, 3, 3, 8, 13, 2, 9], seed=4), 2.5, 30, 1),
    ("restart_5", lambda: Mesh.structured(12, 16), 2.5, 5, 1),
    ("two_sweeps", lambda: Mesh.structured(20, 24), 3.0, 10, 2),
    ("one_line", lambda: Mesh.structured(1, 37), 4.0, 30, 1),
]


@pytest.mark.parametrize("name,mk,shift,restart,ps", CASES, ids=[c[0] for c in CASES])
def test_gmres_matches_oracle(solver, name, mk, shift, restart, ps):
    mesh = mk()
    jac = Jacobian.generate(mesh, shift, 3)
    setup(solver, mesh, jac)
    tol = 1e-10
    it, h = solver.gmres(tol, restart=restart, precond_sweeps=ps, max_iters=300)
    r = oracle.gmres(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, restart, ps, tol, 300,
                     threads=4)
    assert it == r["iters"]
    np.testing.assert_allclose(h, r["hist"], rtol=0, atol=1e-9 * r["hist"][0])
    U = solver.solution()
    assert np.linalg.norm(U - r["U"]) <= 1e-9 * np.linalg.norm(r["U"])
    assert solver.true_residual_norm() <= 1.0000001 * tol * h[0]


def test_gmres_where_line_sweeps_stall(solver):
    """A weak diagonal: plain sweeps make no progress in 300 sweeps while
    GMRES over the same sweep converges."""
    mesh = Mesh.structured(12, 16)
    jac = Jacobian.generate(mesh, 2.0, 2)
    setup(solver, mesh, jac)
    n, h = solver.solve(1e-10, 300)
    assert h[-1] > 1e-10 * h[0]
    it, hg = solver.gmres(1e-10, restart=60, max_iters=300)
    assert hg[-1] <= 1e-10 * hg[0]
    assert solver.true_residual_norm() <= 1.0000001e-10 * hg[0]


def test_gmres_larger_mesh_converges(solver):
    # (at shift 2.5 this mesh makes restarted GMRES(30) stagnate near 7e-3,
    # the oracle's GMRES exactly the same way)
    mesh = Mesh.structured(120, 128)
    jac = Jacobian.generate(mesh, 3.0, 7)
    setup(solver, mesh, jac)
    it, h = solver.gmres(1e-10, restart=30, max_iters=400)
    assert h[-1] <= 1e-10 * h[0]
    assert solver.true_residual_norm() <= 1.0000001e-10 * h[0]
    # deterministic: a second run repeats the history exactly
    it2, h2 = solver.gmres(1e-10, restart=30, max_iters=400)
    assert it2 == it
    np.testing.assert_array_equal(h2, h)


def test_gmres_zero_rhs_and_limits(solver):
    mesh = Mesh.structured(6, 8)
    jac = Jacobian.generate(mesh, 9.0, 1)
    setup(solver, mesh, jac)
    it, h = solver.gmres(1e-12, max_iters=0)
    assert it == 0 and h.size == 1
    it, h = solver.gmres(1e-30, restart=3, max_iters=5)
    assert it == 5
    solver.set_rhs(np.zeros(9 * mesh.nelem))
    it, h = solver.gmres(1e-12)
    assert it == 0 and h[0] == 0.0 and not solver.solution().any()


def test_gmres_errors(solver):
    mesh = Mesh.structured(6, 8)
    jac = Jacobian.generate(mesh, 9.0, 1)
    solver.set_mesh(mesh)
    solver.set_jacobian(jac)
    with pytest.raises(TbsError):
        solver.gmres(1e-10)  # not factored
    solver.factor(ALGO_MIXED)
    with pytest.raises(TbsError):
        solver.gmres(1e-10)  # needs the FP64 line factors
    solver.factor(ALGO_FP64)
    with pytest.raises(TbsError):
        solver.gmres(1e-10, restart=0)
    with pytest.raises(TbsError):
        solver.gmres(1e-10, restart=65)
