"""TBS_ALGO_FP64 for block sizes other than 9 (kernels_nv.cu) on the GPU.

The reference's block-size study (Jacobian::resizeBlockSize,
src/Jacobian.cxx:153-238; the paper's Fig. 8) runs the LIJ sweep at other
nvar.  The general-size kernels run the FP64 form's algorithm, so they are
held to the FP64 bar against the oracle (which is generic in nvar): every
sweep's norm within 1e-12 ||R_0|| of the oracle's, the solution within
1e-12 (relative), the same sweep count to a tolerance.
"""
import numpy as np
import pytest

import oracle
from meshes import ragged_mesh
from triblocksolve_b200 import ALGO_FP64, ALGO_MIXED, ALGO_PIJ, ALGO_REFERENCE, Jacobian, Mesh, Solver
from triblocksolve_b200._native import TbsError

pytestmark = pytest.mark.gpu

SIZES = [2, 3, 4, 5, 7, 8, 10, 12, 16]


@pytest.fixture
def solver():
    s = Solver(0)
    yield s
    s.close()


def setup(s, mesh, jac, algo=ALGO_FP64):
    s.set_mesh(mesh)
    s.set_jacobian(jac)
    s.factor(algo)


def check_sweeps(s, mesh, jac, counts=(1, 2, 4)):
    done = 0
    for n in counts:
        h = s.sweep(n)
        done += n
        r = oracle.lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, done, threads=4)
        r0 = r["hist"][0]
        np.testing.assert_allclose(h, r["hist"][done - n:], rtol=0, atol=1e-12 * r0)
        assert np.linalg.norm(s.solution() - r["U"]) <= 1e-12 * np.linalg.norm(r["U"])
        np.testing.assert_allclose(s.residual(), r["R"], rtol=0, atol=1e-12 * r0)
        np.testing.assert_allclose(s.update(), r["dU"], rtol=0, atol=1e-12 * np.abs(r["U"]).max())


@pytest.mark.parametrize("nv", SIZES)
def test_structured_matches_oracle(solver, nv):
    mesh = Mesh.structured(12, 16, nvar=nv)
    jac = Jacobian.generate(mesh, float(max(9, nv)), 1 + nv)
    setup(solver, mesh, jac)
    check_sweeps(solver, mesh, jac)


@pytest.mark.parametrize("nv", [3, 5, 12])
def test_ragged_matches_oracle(solver, nv):
    mesh = ragged_mesh([5, 1, 7, 3, 3, 8, 13, 2, 9], seed=4, nvar=nv)
    jac = Jacobian.generate(mesh, float(max(9, nv)), 2)
    setup(solver, mesh, jac)
    check_sweeps(solver, mesh, jac)


@pytest.mark.parametrize("nv", [4, 16])
def test_single_line_and_single_cells(solver, nv):
    for mesh in (Mesh.structured(1, 37, nvar=nv), Mesh.structured(6, 1, nvar=nv)):
        jac = Jacobian.generate(mesh, float(max(9, nv)), 3)
        setup(solver, mesh, jac)
        check_sweeps(solver, mesh, jac, counts=(1, 2))


@pytest.mark.parametrize("nv", [5, 10])
def test_solve_sweep_count(solver, nv):
    mesh = Mesh.structured(40, 48, nvar=nv)
    jac = Jacobian.generate(mesh, float(max(6, nv)) - 1.0, 5)
    setup(solver, mesh, jac)
    tol = 1e-11
    n, h = solver.solve(tol, 200)
    r = oracle.lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, 60, threads=4)
    rel = r["hist"] / r["hist"][0]
    assert n == int(np.argmax(rel <= tol))
    np.testing.assert_allclose(h, r["hist"][: n + 1], rtol=0, atol=1e-12 * r["hist"][0])
    assert solver.true_residual_norm() <= 1.0000001 * tol * h[0]
    n2, h2 = solver.solve(tol, 200)
    assert n2 == n
    np.testing.assert_array_equal(h2, h)


def test_from_initial_solution(solver):
    mesh = ragged_mesh([4, 9, 2, 6, 7], seed=8, nvar=6)
    jac = Jacobian.generate(mesh, 9.0, 4)
    U0 = np.random.default_rng(2).uniform(-1, 1, 6 * mesh.nelem)
    setup(solver, mesh, jac)
    solver.set_initial(U0)
    h = solver.sweep(4)
    ref = Solver(0)
    try:
        setup(ref, mesh, jac, ALGO_REFERENCE)
        ref.set_initial(U0)
        hr = ref.sweep(4)
        Ur = ref.solution()
    finally:
        ref.close()
    np.testing.assert_allclose(h, hr, rtol=0, atol=1e-12 * hr[0])
    assert np.linalg.norm(solver.solution() - Ur) <= 1e-12 * np.linalg.norm(Ur)


@pytest.mark.parametrize("nv", [4, 5, 7])
def test_resized_jacobian(solver, nv):
    """The reference's block-size study: a size-9 Jacobian resized by
    resizeBlockSize (new diagonals 10.0, stale leading data kept)."""
    mesh = Mesh.structured(10, 12)
    jac = Jacobian.generate(mesh, 9.0, 6)
    jac.resizeBlockSize(nv)
    mesh.nvar = nv
    setup(solver, mesh, jac)
    h = solver.sweep(3)
    r = oracle.lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, 3, threads=4)
    np.testing.assert_allclose(h, r["hist"], rtol=0, atol=1e-12 * r["hist"][0])
    assert np.linalg.norm(solver.solution() - r["U"]) <= 1e-12 * np.linalg.norm(r["U"])


def test_grown_jacobian_fails_loudly(solver):
    """Growing the blocks puts 10.0 on the diagonals of the face blocks too,
    which makes the line pivots singular: the reference's own sweep turns
    to NaN, the FP64 factorization reports TBS_ERR_NUMERIC."""
    mesh = Mesh.structured(10, 12)
    jac = Jacobian.generate(mesh, 9.0, 6)
    jac.resizeBlockSize(12)
    mesh.nvar = 12
    r = oracle.lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, 1)
    assert not np.isfinite(r["hist"][1])
    solver.set_mesh(mesh)
    solver.set_jacobian(jac)
    with pytest.raises(TbsError) as e:
        solver.factor(ALGO_FP64)
    assert e.value.code == 6  # TBS_ERR_NUMERIC


def test_size9_only_forms_refuse_other_sizes(solver):
    mesh = Mesh.structured(6, 8, nvar=5)
    jac = Jacobian.generate(mesh, 9.0, 1)
    solver.set_mesh(mesh)
    solver.set_jacobian(jac)
    for algo in (ALGO_MIXED, ALGO_PIJ):
        with pytest.raises(TbsError):
            solver.factor(algo)
    solver.factor(ALGO_FP64)
    with pytest.raises(TbsError):
        solver.solve_multi(np.zeros((2, 5 * mesh.nelem)), 1e-10, 10)
    with pytest.raises(TbsError):
        solver.gmres(1e-10)
    big = Mesh.structured(2, 3, nvar=17)
    s2 = Solver(0)
    try:
        s2.set_mesh(big)
        s2.set_jacobian(Jacobian.generate(big, 20.0, 1))
        with pytest.raises(TbsError):
            s2.factor(ALGO_FP64)
        s2.factor(ALGO_REFERENCE)  # the reference order covers every size
    finally:
        s2.close()
