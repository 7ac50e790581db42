"""The true-residual check of tbs_solve, and a lagged factorization
(tbs_update_values), through the C ABI.

TBS_ALGO_FP64 tracks its residual recursively.  When that residual meets the
tolerance, tbs_solve recomputes rhs + J U from the original blocks (the rule
of linesmoothLU_TriBlock_v3.okl:228-336) and either ends the solve or goes
on from the true residual.  The drift case is made on the host, with no
fault: new block values after the factorization make the factored system
differ from the true one, so the recursive residual converges to the old
system and the check must catch it.

Tolerances: a reported convergence has a true relative residual at or
below the tolerance (1.0000001 x, for the norm's last rounding); solutions
of the new system within 1e-9 (relative) of the oracle's, run on the new
values to 1e-14.
"""
import numpy as np
import pytest

import oracle
from meshes import ragged_mesh
from triblocksolve_b200 import (ALGO_FP64, ALGO_MIXED, ALGO_PIJ, ALGO_REFERENCE, Batch, Jacobian,
                                Mesh, Solver, TbsError)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solver():
    s = Solver(0)
    yield s
    s.set_check(True)
    s.close()


def perturbed(jac, seed, scale):
    """The Jacobian with every block entry moved by scale * U(-1,1) * |entry|."""
    rng = np.random.default_rng(seed)
    out = []
    for a in (jac.jacD, jac.jacO1, jac.jacO2):
        out.append(a * (1.0 + scale * rng.uniform(-1.0, 1.0, a.size)))
    return out


def oracle_solution(mesh, D, O1, O2, rhs):
    r = oracle.lij(mesh, D, O1, O2, rhs, 40, threads=4)
    return r["U"]


def test_converged_solve_is_checked(solver):
    mesh = Mesh.structured(60, 64)
    jac = Jacobian.generate(mesh, 9.0, 1)
    solver.set_mesh(mesh)
    solver.set_jacobian(jac)
    solver.factor(ALGO_FP64)
    n, h = solver.solve(1e-12, 100)
    tn, checks, restarts = solver.solve_check()
    assert checks == 1 and restarts == 0
    assert tn <= 1e-12 * h[0] * 1.0000001
    assert tn == pytest.approx(solver.true_residual_norm(), rel=1e-12)
    # the check leaves the history of an unperturbed solve unchanged
    ref = oracle.lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, n, threads=4)
    assert np.all(np.abs(h - ref["hist"]) <= 1e-12 * ref["hist"][0])
    # with the check off, the same sweeps and history, no check recorded
    solver.set_check(False)
    n2, h2 = solver.solve(1e-12, 100)
    assert n2 == n
    np.testing.assert_array_equal(h2, h)
    assert solver.solve_check()[1] == 0
    solver.set_check(True)


@pytest.mark.parametrize("profiled", [False, True])
def test_drift_is_caught_fp64(solver, profiled):
    """Factored on old values, residual on new ones: the recursive residual
    converges to the old system, the check restarts it until the new system
    is solved.  The eager (profiled) solve makes the same decisions."""
    mesh = Mesh.structured(30, 40)
    jac = Jacobian.generate(mesh, 9.0, 3)
    D, O1, O2 = perturbed(jac, 5, 0.02)
    solver.set_mesh(mesh)
    solver.set_jacobian(jac)
    solver.factor(ALGO_FP64)
    solver.update_values(D, O1, O2)
    solver.profile(profiled)
    n, h = solver.solve(1e-10, 200)
    solver.profile(False)
    tn, checks, restarts = solver.solve_check()
    true_rel = solver.true_residual_norm() / h[0]
    print(f"fp64 drift: {n} sweeps, {checks} checks, {restarts} restarts, true rel {true_rel:.2e}")
    assert restarts >= 1 and checks == restarts + 1
    assert h[-1] <= 1e-10 * h[0] and true_rel <= 1e-10 * 1.0000001
    U_new = oracle_solution(mesh, D, O1, O2, jac.rhs)
    assert np.linalg.norm(solver.solution() - U_new) <= 1e-9 * np.linalg.norm(U_new)
    # without the update the old system's solution differs by far more
    U_old = oracle_solution(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs)
    assert np.linalg.norm(U_old - U_new) > 1e-4 * np.linalg.norm(U_new)


def test_drift_graph_and_eager_agree(solver):
    mesh = ragged_mesh([9, 4, 12, 7, 3, 10], seed=5)
    jac = Jacobian.generate(mesh, 9.0, 6)
    D, O1, O2 = perturbed(jac, 8, 0.03)
    solver.set_mesh(mesh)
    solver.set_jacobian(jac)
    solver.factor(ALGO_FP64)
    solver.update_values(D, O1, O2)
    n1, h1 = solver.solve(1e-11, 200)
    c1 = solver.solve_check()
    U1 = solver.solution()
    solver.profile(True)
    n2, h2 = solver.solve(1e-11, 200)
    solver.profile(False)
    assert n2 == n1 and solver.solve_check() == c1
    np.testing.assert_array_equal(h2, h1)
    np.testing.assert_array_equal(solver.solution(), U1)


def test_drift_at_the_sweep_limit_reports_the_true_norm(solver):
    """A failed check at the last allowed sweep ends the solve with the true
    residual's norm as the last history entry: no false convergence."""
    mesh = Mesh.structured(20, 24)
    jac = Jacobian.generate(mesh, 9.0, 9)
    D, O1, O2 = perturbed(jac, 10, 0.05)
    solver.set_mesh(mesh)
    solver.set_jacobian(jac)
    solver.factor(ALGO_FP64)
    solver.update_values(D, O1, O2)
    # the smallest sweep limit at which the old system's recursion passes
    first = None
    for limit in range(1, 60):
        n, h = solver.solve(1e-10, limit)
        tn, checks, restarts = solver.solve_check()
        if checks >= 1:
            first = limit
            break
    assert first is not None
    assert restarts == 1 and h[-1] == tn and h[-1] > 1e-10 * h[0]
    assert n == first


def test_reference_and_mixed_follow_new_values(solver):
    mesh = Mesh.structured(24, 30)
    jac = Jacobian.generate(mesh, 6.0, 12)
    D, O1, O2 = perturbed(jac, 13, 0.02)
    U_new = oracle_solution(mesh, D, O1, O2, jac.rhs)
    for algo in (ALGO_REFERENCE, ALGO_MIXED):
        solver.set_mesh(mesh)
        solver.set_jacobian(jac)
        solver.factor(algo)
        solver.update_values(D, O1, O2)
        n, h = solver.solve(1e-10, 300)
        assert h[-1] <= 1e-10 * h[0]
        assert solver.true_residual_norm() <= 1e-10 * h[0] * 1.0000001
        assert np.linalg.norm(solver.solution() - U_new) <= 1e-9 * np.linalg.norm(U_new)


def test_check_at_block_size_5(solver):
    mesh = Mesh.structured(16, 20, nvar=5)
    jac = Jacobian.generate(mesh, 5.0, 14)
    D, O1, O2 = perturbed(jac, 15, 0.02)
    solver.set_mesh(mesh)
    solver.set_jacobian(jac)
    solver.factor(ALGO_FP64)
    n, h = solver.solve(1e-12, 100)
    assert solver.solve_check()[1:] == (1, 0)
    solver.update_values(D, O1, O2)
    n, h = solver.solve(1e-10, 300)
    tn, checks, restarts = solver.solve_check()
    assert restarts >= 1
    assert solver.true_residual_norm() <= 1e-10 * h[0] * 1.0000001
    U_new = oracle_solution(mesh, D, O1, O2, jac.rhs)
    assert np.linalg.norm(solver.solution() - U_new) <= 1e-9 * np.linalg.norm(U_new)


def test_update_values_refusals(solver):
    mesh = Mesh.structured(8, 10)
    jac = Jacobian.generate(mesh, 9.0, 16)
    solver.set_mesh(mesh)
    solver.set_jacobian(jac)
    solver.factor(ALGO_PIJ)
    with pytest.raises(TbsError):
        solver.update_values(jac.jacD, jac.jacO1, jac.jacO2)
    solver.factor(ALGO_FP64)
    solver.set_check(False)
    with pytest.raises(TbsError):
        solver.update_values(jac.jacD, jac.jacO1, jac.jacO2)
    solver.set_check(True)
    solver.update_values(jac.jacD, jac.jacO1, jac.jacO2)  # same values: an ordinary solve
    n, h = solver.solve(1e-12, 100)
    assert solver.solve_check()[1:] == (1, 0)
    # the paths that track the residual with the factorization's blocks refuse
    # a context whose values are newer than its factorization, until it is re-factored
    with pytest.raises(TbsError):
        solver.solve_multi(np.stack([jac.rhs, jac.rhs]), 1e-10, 50)
    with pytest.raises(TbsError):
        solver.gmres(1e-10, 10, 1, 50)
    with pytest.raises(TbsError):
        b = Batch([solver])
        try:
            b.solve(1e-10, 50)
        finally:
            b.close()
    solver.factor(ALGO_FP64)
    solver.solve_multi(np.stack([jac.rhs, jac.rhs]), 1e-10, 50)
    solver.gmres(1e-10, 10, 1, 50)
