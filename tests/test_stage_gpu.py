"""tbs_stage_jacobian: the next system's Jacobian uploaded on the copy
stream while the current one is solved, switched in by tbs_factor.

Every result of a staged pipeline must be bit-identical to the same system
set with tbs_set_jacobian and solved alone (the same kernels on the same
values), for the FP64, mixed and reference-order algorithms, with one solve
graph reused across switches (the first stage, with no active set yet,
adopts the landing buffers; later ones are copied over the active set); a
batch over a context that switched sets must see the new values.
"""
import numpy as np
import pytest
import torch

from meshes import ragged_mesh
from triblocksolve_b200 import ALGO_FP64, ALGO_MIXED, ALGO_REFERENCE, Batch, Jacobian, Mesh, Solver
from triblocksolve_b200._native import TbsError

pytestmark = pytest.mark.gpu


def pinned(a):
    t = torch.empty(a.size, dtype=torch.float64, pin_memory=True).numpy()
    t[:] = a
    return t


def systems(mesh, n, shift=6.0):
    out = []
    for k in range(n):
        j = Jacobian.generate(mesh, shift, 100 + k)
        out.append(tuple(pinned(a) for a in (j.jacD, j.jacO1, j.jacO2, j.rhs)))
    return out


def alone(mesh, sysk, algo, tol):
    s = Solver(0)
    s.set_mesh(mesh)
    s.set_jacobian_arrays(*sysk)
    s.factor(algo)
    n, h = s.solve(tol, 200)
    U = s.solution()
    s.close()
    return n, h, U


@pytest.mark.parametrize("algo,tol", [(ALGO_FP64, 1e-12), (ALGO_MIXED, 1e-10),
                                      (ALGO_REFERENCE, 1e-10)])
def test_staged_pipeline_equals_alone(algo, tol):
    mesh = Mesh.structured(30, 40)
    syss = systems(mesh, 4)
    want = [alone(mesh, sk, algo, tol) for sk in syss]
    s = Solver(0)
    s.set_mesh(mesh)
    s.stage_jacobian_arrays(*syss[0])       # no tbs_set_jacobian before it
    s.factor(algo)
    for k in range(len(syss)):
        if k + 1 < len(syss):
            s.stage_jacobian_arrays(*syss[k + 1])   # uploads while system k is solved
        n, h = s.solve(tol, 200)
        U = s.solution()
        assert n == want[k][0], k
        np.testing.assert_array_equal(h, want[k][1])
        np.testing.assert_array_equal(U, want[k][2])
        if k + 1 < len(syss):
            s.factor(algo)
    # a second pass repeats it with the solve graph already built
    s.stage_jacobian_arrays(*syss[1])
    s.factor(algo)
    n, h = s.solve(tol, 200)
    np.testing.assert_array_equal(s.solution(), want[1][2])
    s.close()


@pytest.mark.parametrize("algo,tol", [(ALGO_FP64, 1e-12), (ALGO_MIXED, 1e-10)])
def test_two_staged_ahead_equals_alone(algo, tol):
    """Two systems staged before the first factorization, then one staged
    two ahead of the solve each step (both landing slots in turn), as the
    bench's stream of systems runs it; a third stage is refused."""
    mesh = Mesh.structured(24, 36)
    syss = systems(mesh, 5, shift=7.0)
    want = [alone(mesh, sk, algo, tol) for sk in syss]
    s = Solver(0)
    s.set_mesh(mesh)
    s.set_jacobian_arrays(*syss[4])          # an active set that the stream replaces
    s.factor(algo)
    s.solve(tol, 200)
    s.stage_jacobian_arrays(*syss[0])
    s.stage_jacobian_arrays(*syss[1])
    with pytest.raises(TbsError):
        s.stage_jacobian_arrays(*syss[2])
    s.factor(algo)
    for k in range(len(syss)):
        n, h = s.solve(tol, 200)
        U = s.solution()
        assert n == want[k][0], k
        np.testing.assert_array_equal(h, want[k][1])
        np.testing.assert_array_equal(U, want[k][2])
        if k + 2 < len(syss):
            s.stage_jacobian_arrays(*syss[k + 2])
        if k + 1 < len(syss):
            s.factor(algo)
    s.close()


def test_set_jacobian_discards_a_staged_set():
    mesh = ragged_mesh([7, 3, 9, 5, 2], seed=3)
    syss = systems(mesh, 2, shift=9.0)
    want = alone(mesh, syss[1], ALGO_FP64, 1e-12)
    s = Solver(0)
    s.set_mesh(mesh)
    s.stage_jacobian_arrays(*syss[0])
    s.set_jacobian_arrays(*syss[1])          # these values win
    s.factor(ALGO_FP64)
    n, h = s.solve(1e-12, 200)
    assert n == want[0]
    np.testing.assert_array_equal(s.solution(), want[2])
    s.close()


def test_batch_follows_a_switched_set():
    mesh = Mesh.structured(12, 20)
    syss = systems(mesh, 2, shift=9.0)
    want = alone(mesh, syss[1], ALGO_FP64, 1e-12)
    s = Solver(0)
    s.set_mesh(mesh)
    s.set_jacobian_arrays(*syss[0])
    s.factor(ALGO_FP64)
    b = Batch([s])
    b.solve(1e-12, 200)
    s.stage_jacobian_arrays(*syss[1])
    s.factor(ALGO_FP64)
    sw, hist = b.solve(1e-12, 200)
    assert int(sw[0]) == want[0]
    np.testing.assert_array_equal(s.solution(), want[2])
    b.close()
    s.close()
