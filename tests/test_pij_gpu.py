"""Point-implicit Jacobi (TBS_ALGO_PIJ) on the GPU.

The oracle is the reference's own line sweep on the same mesh with every
cell its own line (oracle.pij), which tests/test_oracle.py pins to a dense
statement of the PIJ iteration.  TBS_ALGO_PIJ updates the residual from the
face couplings (R_new = sum offJ dU_nbr, exact for an exact point solve) and
multiplies by an explicit D^-1, so like TBS_ALGO_FP64 it is held to
| ||R_k|| - ||R_k||_oracle | <= 1e-12 ||R_0|| on every sweep and
||U - U_oracle|| <= 1e-12 ||U_oracle||.  TBS_ALGO_REFERENCE run on the
one-cell-line mesh is the same iteration in the reference's operation order
and must equal the oracle bit for bit.
"""
import numpy as np
import pytest

import oracle
from meshes import point_mesh, ragged_mesh
from triblocksolve_b200 import ALGO_PIJ, ALGO_REFERENCE, Jacobian, Mesh, Solver
from triblocksolve_b200._native import TbsError

pytestmark = pytest.mark.gpu

CASES = {
    "structured_20x24": lambda: Mesh.structured(20, 24),
    "ragged": lambda: ragged_mesh([5, 1, 7, 3, 3, 8, 13, 2, 9], seed=4),
    "one_line": lambda: Mesh.structured(1, 37),
    "one_cell_lines": lambda: Mesh.structured(6, 1),
    "single_cell": lambda: Mesh.structured(1, 1),
    "structured_60x64": lambda: Mesh.structured(60, 64),
}


@pytest.fixture
def solver():
    s = Solver(0)
    yield s
    s.close()


def setup(s, mesh, jac, algo):
    s.set_mesh(mesh)
    s.set_jacobian(jac)
    s.factor(algo)


@pytest.mark.parametrize("case", list(CASES))
def test_pij_sweeps_match_oracle(solver, case):
    mesh = CASES[case]()
    jac = Jacobian.generate(mesh, 9.0, 2)
    setup(solver, mesh, jac, ALGO_PIJ)
    done = 0
    for n in (1, 2, 5):
        h = solver.sweep(n)
        done += n
        r = oracle.pij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, done, threads=4)
        r0 = r["hist"][0]
        np.testing.assert_allclose(h, r["hist"][done - n:], rtol=0, atol=1e-12 * r0)
        U = solver.solution()
        assert np.linalg.norm(U - r["U"]) <= 1e-12 * max(np.linalg.norm(r["U"]), 1e-300)
        np.testing.assert_allclose(solver.update(), r["dU"], rtol=0,
                                   atol=1e-12 * max(np.abs(r["U"]).max(), 1e-300))
        np.testing.assert_allclose(solver.residual(), r["R"], rtol=0, atol=1e-12 * r0)


@pytest.mark.parametrize("case", ["structured_20x24", "ragged", "one_line"])
def test_reference_order_on_one_cell_lines_is_bit_exact(solver, case):
    mesh = CASES[case]()
    pm = point_mesh(mesh)
    jac = Jacobian.generate(mesh, 9.0, 3)
    setup(solver, pm, jac, ALGO_REFERENCE)
    solver.sweep(6)
    r = oracle.pij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, 6, threads=4)
    np.testing.assert_array_equal(solver.solution(), r["U"])
    np.testing.assert_array_equal(solver.residual(), r["R"])


@pytest.mark.parametrize("tol", [1e-6, 1e-12])
def test_pij_solve_sweep_count(solver, tol):
    mesh = Mesh.structured(60, 64)
    jac = Jacobian.generate(mesh, 9.0, 1)
    setup(solver, mesh, jac, ALGO_PIJ)
    sweeps, h = solver.solve(tol, 400)
    r = oracle.pij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, 80, threads=4)
    rel = r["hist"] / r["hist"][0]
    want = int(np.argmax(rel <= tol))
    assert sweeps == want
    assert np.all(np.abs(h - r["hist"][: sweeps + 1]) <= 1e-12 * r["hist"][0])
    assert solver.true_residual_norm() <= 1.0000001 * tol * h[0]
    # a second solve repeats the history exactly (the update buffers'
    # parity restarts with the solve)
    s2, h2 = solver.solve(tol, 400)
    assert s2 == sweeps
    np.testing.assert_array_equal(h2, h)


def test_pij_sweep_parity_across_calls(solver):
    """Odd sweep counts across tbs_sweep calls and a solve in between: the
    swapping update buffers must keep U and the norms on the oracle."""
    mesh = ragged_mesh([4, 9, 2, 6, 7], seed=8)
    jac = Jacobian.generate(mesh, 6.0, 4)
    setup(solver, mesh, jac, ALGO_PIJ)
    solver.solve(1e-8, 100)
    solver.set_rhs(jac.rhs)
    done = 0
    for n in (3, 1, 3):
        solver.sweep(n)
        done += n
    r = oracle.pij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, done)
    assert np.linalg.norm(solver.solution() - r["U"]) <= 1e-12 * np.linalg.norm(r["U"])


def test_pij_from_initial_solution(solver):
    mesh = Mesh.structured(12, 20)
    jac = Jacobian.generate(mesh, 9.0, 5)
    rng = np.random.default_rng(1)
    U0 = rng.uniform(-1, 1, 9 * mesh.nelem)
    setup(solver, mesh, jac, ALGO_PIJ)
    solver.set_initial(U0)
    solver.sweep(4)
    U = solver.solution()
    # the same iteration in reference order from the same start
    ref = Solver(0)
    try:
        setup(ref, point_mesh(mesh), jac, ALGO_REFERENCE)
        ref.set_initial(U0)
        ref.sweep(4)
        Ur = ref.solution()
    finally:
        ref.close()
    assert np.linalg.norm(U - Ur) <= 1e-12 * np.linalg.norm(Ur)


def test_pij_zero_pivot_reported(solver):
    mesh = Mesh.structured(4, 5)
    jac = Jacobian.generate(mesh, 9.0, 1)
    jac.jacD[81 * 7: 81 * 8] = 0.0  # one singular diagonal block
    solver.set_mesh(mesh)
    solver.set_jacobian(jac)
    with pytest.raises(TbsError):
        solver.factor(ALGO_PIJ)
