"""GPU parity against the CPU oracle, through the C ABI.

Tolerances (stated per algorithm):
  TBS_ALGO_REFERENCE  bit-identical U, R, dU after every sweep (same
                      operation order, no FMA contraction on either side).
  TBS_ALGO_FP64       per-sweep | ||R_k|| - ||R_k||_oracle | <= 1e-12 ||R_0||,
                      ||U - U_oracle|| <= 1e-12 ||U_oracle||, the same sweep
                      count at a tolerance.
  TBS_ALGO_MIXED      reaches 1e-10 true relative residual; solution within
                      1e-9 (relative) of the FP64 oracle's converged solution.
"""
import numpy as np
import pytest

import oracle
from meshes import ragged_mesh
from triblocksolve_b200 import ALGO_FP64, ALGO_MIXED, ALGO_REFERENCE, Jacobian, Mesh, Solver

pytestmark = pytest.mark.gpu

CASES = {
    "60x64": lambda: Mesh.structured(60, 64),
    "ragged": lambda: ragged_mesh([5, 1, 7, 3, 3, 8, 13, 2, 9], seed=4),
    "single_line": lambda: Mesh.structured(1, 37),
    "single_cells": lambda: Mesh.structured(6, 1),
    "one_cell": lambda: Mesh.structured(1, 1),
    "odd_lines": lambda: Mesh.structured(7, 11),
}


@pytest.fixture(scope="module")
def solver():
    s = Solver(0)
    yield s
    s.close()


def setup(solver, mesh, jac, algo):
    solver.set_mesh(mesh)
    solver.set_jacobian(jac)
    solver.factor(algo)


@pytest.mark.parametrize("case", list(CASES))
def test_reference_algo_bit_exact(solver, case):
    mesh = CASES[case]()
    jac = Jacobian.generate(mesh, 9.0, 1)
    setup(solver, mesh, jac, ALGO_REFERENCE)
    done = 0
    for n in (1, 1, 3):
        solver.sweep(n)
        done += n
        r = oracle.lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, done, threads=4)
        np.testing.assert_array_equal(solver.solution(), r["U"])
        np.testing.assert_array_equal(solver.residual(), r["R"])
        np.testing.assert_array_equal(solver.update(), r["dU"])


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("case", list(CASES) + ["nvar5"])
def test_reference_algo_equals_reference_kernels(solver, case):
    """TBS_ALGO_REFERENCE against the reference's own kernels (OKL translated
    to C, oracle/_ref): U, R and dU bit for bit after every sweep."""
    mesh = Mesh.structured(12, 16, nvar=5) if case == "nvar5" else CASES[case]()
    jac = Jacobian.generate(mesh, 9.0, 11)
    setup(solver, mesh, jac, ALGO_REFERENCE)
    n = 6
    r = oracle.ref_lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, n, threads=4, per_sweep=True)
    for p in range(n):
        solver.sweep(1)
        np.testing.assert_array_equal(solver.solution(), r["U_all"][p])
        np.testing.assert_array_equal(solver.residual(), r["R_all"][p])
        np.testing.assert_array_equal(solver.update(), r["dU_all"][p])


def test_reference_algo_generic_block_size(solver):
    mesh = ragged_mesh([4, 6, 2, 5], seed=2, nvar=5)
    jac = Jacobian.generate(mesh, 5.0, 6)
    setup(solver, mesh, jac, ALGO_REFERENCE)
    h = solver.sweep(6)
    r = oracle.lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, 6)
    np.testing.assert_array_equal(solver.solution(), r["U"])
    np.testing.assert_array_equal(solver.residual(), r["R"])
    np.testing.assert_allclose(h, r["hist"], rtol=1e-14, atol=0)


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("shift", [9.0, 4.0])
def test_fp64_algo_within_tolerance(solver, case, shift):
    mesh = CASES[case]()
    jac = Jacobian.generate(mesh, shift, 2)
    setup(solver, mesh, jac, ALGO_FP64)
    n = 12
    h = solver.sweep(n)
    r = oracle.lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, n, threads=4)
    r0 = r["hist"][0]
    assert np.all(np.abs(h - r["hist"]) <= 1e-12 * r0), (h, r["hist"])
    U = solver.solution()
    assert np.linalg.norm(U - r["U"]) <= 1e-12 * np.linalg.norm(r["U"])
    # the recursive residual and the recomputed true residual agree
    R = solver.residual()
    np.testing.assert_allclose(R, oracle.true_residual(mesh, jac.jacD, jac.jacO1, jac.jacO2,
                                                       jac.rhs, U), rtol=0, atol=1e-13 * r0)
    assert abs(solver.true_residual_norm() - np.linalg.norm(R)) <= 1e-13 * r0


@pytest.mark.parametrize("algo", [ALGO_REFERENCE, ALGO_FP64])
@pytest.mark.parametrize("tol", [1e-6, 1e-12])
def test_solve_sweep_count_matches_oracle(solver, algo, tol):
    mesh = Mesh.structured(60, 64)
    jac = Jacobian.generate(mesh, 9.0, 1)
    setup(solver, mesh, jac, algo)
    sweeps, h = solver.solve(tol, 200)
    r = oracle.lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, 40, threads=4)
    rel = r["hist"] / r["hist"][0]
    want = int(np.argmax(rel <= tol))
    assert sweeps == want
    assert np.all(np.abs(h - r["hist"][: sweeps + 1]) <= 1e-12 * r["hist"][0])
    # a second solve restarts from U = 0 and repeats the history exactly
    s2, h2 = solver.solve(tol, 200)
    assert s2 == sweeps
    np.testing.assert_array_equal(h2, h)


def test_solve_respects_sweep_limit(solver):
    mesh = Mesh.structured(20, 24)
    jac = Jacobian.generate(mesh, 9.0, 3)
    setup(solver, mesh, jac, ALGO_FP64)
    s, h = solver.solve(1e-30, 5)
    assert s == 5 and h.size == 6
    s, h = solver.solve(1e-12, 0)
    assert s == 0 and h.size == 1


def test_mixed_reaches_1e10(solver):
    mesh = Mesh.structured(60, 64)
    jac = Jacobian.generate(mesh, 4.0, 5)
    setup(solver, mesh, jac, ALGO_MIXED)
    sweeps, h = solver.solve(1e-10, 50)
    assert h[-1] <= 1e-10 * h[0]
    r = oracle.lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, 30, threads=4)
    U = solver.solution()
    assert np.linalg.norm(U - r["U"]) <= 1e-9 * np.linalg.norm(r["U"])
    assert solver.true_residual_norm() <= 1.0000001e-10 * h[0]


def test_repeated_rhs_and_restart(solver):
    mesh = ragged_mesh([8, 3, 8, 6, 2], seed=9)
    jac = Jacobian.generate(mesh, 9.0, 4)
    setup(solver, mesh, jac, ALGO_FP64)
    rng = np.random.default_rng(0)
    for _ in range(3):
        rhs = rng.uniform(-1, 1, jac.rhs.size)
        solver.set_rhs(rhs)
        h = solver.sweep(6)
        r = oracle.lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, rhs, 6)
        assert np.all(np.abs(h - r["hist"]) <= 1e-12 * r["hist"][0])
        assert np.linalg.norm(solver.solution() - r["U"]) <= 1e-12 * np.linalg.norm(r["U"])


def test_checkpoint_resume(solver):
    """tbs_set_initial: 3 sweeps, checkpoint U, resume for 4 more == 7 straight."""
    mesh = Mesh.structured(10, 12)
    jac = Jacobian.generate(mesh, 9.0, 7)
    for algo in (ALGO_REFERENCE, ALGO_FP64):
        setup(solver, mesh, jac, algo)
        solver.sweep(3)
        U3 = solver.solution()
        solver.set_initial(U3)
        h = solver.sweep(4)
        r = oracle.lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, 7)
        assert np.linalg.norm(solver.solution() - r["U"]) <= 1e-12 * np.linalg.norm(r["U"])
        assert abs(h[-1] - r["hist"][-1]) <= 1e-12 * r["hist"][0]
        solver.set_initial(None)


@pytest.mark.parametrize("case", ["ragged", "single_line", "odd_lines", "single_cells"])
def test_mixed_other_meshes(solver, case):
    mesh = CASES[case]()
    jac = Jacobian.generate(mesh, 6.0, 8)
    setup(solver, mesh, jac, ALGO_MIXED)
    sweeps, h = solver.solve(1e-10, 60)
    assert h[-1] <= 1e-10 * h[0]
    assert solver.true_residual_norm() <= 1.0000001e-10 * h[0]
    r = oracle.lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, 40)
    assert np.linalg.norm(solver.solution() - r["U"]) <= 1e-9 * np.linalg.norm(r["U"])


def test_tune_inner_picks_a_converging_count(solver):
    mesh = Mesh.structured(40, 48)
    jac = Jacobian.generate(mesh, 4.0, 2)
    setup(solver, mesh, jac, ALGO_MIXED)
    m, ms = solver.tune_inner(1e-10, 60)
    assert m in (2, 3, 4, 5, 6, 8, 10) and ms > 0
    sweeps, h = solver.solve(1e-10, 60)
    assert h[-1] <= 1e-10 * h[0]


def test_mixed_inner_schedule(solver):
    """A first outer step with its own inner sweep count: the graph solve,
    the eager (profiled) solve and a tbs_sweep sequence give the same
    iterates, and the solve still reaches the FP64 tolerance."""
    mesh = Mesh.structured(40, 48)
    jac = Jacobian.generate(mesh, 4.0, 3)
    setup(solver, mesh, jac, ALGO_MIXED)
    solver.set_inner_schedule(2, 4)
    assert solver.inner_schedule() == (2, 4)
    n, h = solver.solve(1e-10, 60)
    assert h[-1] <= 1e-10 * h[0]
    U = solver.solution()
    solver.profile(True)
    n2, h2 = solver.solve(1e-10, 60)
    solver.profile(False)
    assert n2 == n
    np.testing.assert_array_equal(h2, h)
    np.testing.assert_array_equal(solver.solution(), U)
    solver.set_rhs(jac.rhs)  # a new start: the next sweep is a first step
    h3 = solver.sweep(n)
    np.testing.assert_array_equal(h3, h)
    np.testing.assert_array_equal(solver.solution(), U)
    # a different first step changes the iterates (the schedule is in effect)
    solver.set_inner_schedule(4, 4)
    _, h4 = solver.solve(1e-10, 60)
    assert h4[1] != h[1]


def test_contexts_of_different_shapes_in_one_process():
    """A kernel's shared-memory limit is one value for the whole process: a
    context with short lines, factored after one with long lines, must not
    lower it under the first one's launches."""
    big_mesh, small_mesh = Mesh.structured(8, 200), Mesh.structured(4, 4)
    big_jac, small_jac = Jacobian.generate(big_mesh, 9.0, 2), Jacobian.generate(small_mesh, 9.0, 3)
    big, small = Solver(0), Solver(0)
    big.set_mesh(big_mesh)
    big.set_jacobian(big_jac)
    big.factor(ALGO_FP64)
    small.set_mesh(small_mesh)
    small.set_jacobian(small_jac)
    small.factor(ALGO_FP64)
    n, h = big.solve(1e-12, 100)
    ref = oracle.lij(big_mesh, big_jac.jacD, big_jac.jacO1, big_jac.jacO2, big_jac.rhs, n)
    assert np.all(np.abs(h - ref["hist"]) <= 1e-12 * ref["hist"][0])
    small.solve(1e-12, 100)
    big.close()
    small.close()
