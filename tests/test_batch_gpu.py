"""Batched solves (tbs_batch_*) on the GPU.

The batch runs the single-system kernels' per-unit arithmetic and norm
order, so every member's sweep count, norm history and solution must be
bit-identical to tbs_solve of that member alone (checked with exact
equality), for both TBS_ALGO_FP64 and TBS_ALGO_MIXED, for any schedule of
the persistent Thomas launch, and with members that converge at different
sweeps, start from tbs_set_initial, or are re-factored between solves.
The alone solves are themselves pinned to the CPU oracle by
test_parity_gpu.py; the FP64 batch is also checked against the oracle here.
"""
import numpy as np
import pytest

import oracle
from meshes import ragged_mesh
from triblocksolve_b200 import ALGO_FP64, ALGO_MIXED, ALGO_REFERENCE, Batch, Jacobian, Mesh, Solver
from triblocksolve_b200._native import TbsError

pytestmark = pytest.mark.gpu

SYSTEMS = [
    (lambda: Mesh.structured(24, 40), 9.0, 1),
    (lambda: ragged_mesh([5, 1, 7, 3, 3, 8, 13, 2, 9], seed=4), 9.0, 2),
    (lambda: Mesh.structured(1, 37), 9.0, 3),
    (lambda: Mesh.structured(6, 1), 9.0, 4),
    (lambda: Mesh.structured(7, 11), 4.0, 5),      # converges later than the others
    (lambda: Mesh.structured(1, 1), 9.0, 6),
    (lambda: Mesh.structured(40, 96), 6.0, 7),
]


def make_members(algo, pick=None):
    out = []
    for k, (mk, shift, seed) in enumerate(SYSTEMS):
        if pick is not None and k not in pick:
            continue
        mesh = mk()
        jac = Jacobian.generate(mesh, shift, seed)
        s = Solver(0)
        s.set_mesh(mesh)
        s.set_jacobian(jac)
        s.factor(algo)
        out.append((s, mesh, jac))
    return out


def close_all(members, batch=None):
    if batch is not None:
        batch.close()
    for s, _, _ in members:
        s.close()


def batch_vs_alone(members, batch, tol, max_sweeps):
    sw, hist = batch.solve(tol, max_sweeps)
    sols = [s.solution() for s, _, _ in members]
    for k, (s, _, _) in enumerate(members):
        n1, h1 = s.solve(tol, max_sweeps)
        assert n1 == sw[k], (k, n1, sw[k])
        np.testing.assert_array_equal(hist[k], h1)
        np.testing.assert_array_equal(sols[k], s.solution())
    return sw, hist


@pytest.mark.parametrize("algo", [ALGO_FP64, ALGO_MIXED])
def test_batch_equals_alone(algo):
    members = make_members(algo)
    b = Batch([m[0] for m in members])
    try:
        tol = 1e-12 if algo == ALGO_FP64 else 1e-10
        sw, hist = batch_vs_alone(members, b, tol, 80)
        assert len(set(int(x) for x in sw)) > 1  # members stop at their own sweep
        for k in range(len(members)):
            assert hist[k][-1] <= tol * hist[k][0]
        # a second batched solve restarts from U = 0 and repeats itself
        sw2, hist2 = b.solve(tol, 80)
        np.testing.assert_array_equal(sw2, sw)
        for k in range(len(members)):
            np.testing.assert_array_equal(hist2[k], hist[k])
    finally:
        close_all(members, b)


def test_batch_fp64_matches_oracle():
    members = make_members(ALGO_FP64, pick={0, 1, 4})
    b = Batch([m[0] for m in members])
    try:
        sw, hist = b.solve(1e-12, 80)
        for k, (s, mesh, jac) in enumerate(members):
            r = oracle.lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, int(sw[k]), threads=4)
            r0 = r["hist"][0]
            assert np.all(np.abs(hist[k] - r["hist"]) <= 1e-12 * r0)
            assert np.linalg.norm(s.solution() - r["U"]) <= 1e-12 * np.linalg.norm(r["U"])
    finally:
        close_all(members, b)


@pytest.mark.parametrize("algo", [ALGO_FP64, ALGO_MIXED])
def test_batch_schedules_agree(algo):
    members = make_members(algo, pick={0, 1, 2, 4, 6})
    b = Batch([m[0] for m in members])
    try:
        tol = 1e-12 if algo == ALGO_FP64 else 1e-10
        sw0, h0 = b.solve(tol, 80)
        u0 = [s.solution() for s, _, _ in members]
        for warps in (1, 2):
            b.set_warps_per_line(warps)
            assert b.warps_per_line() == warps
            for ctas, stages, order in [(1, 2, 0), (3, 3, 1), (2, 4, 0), (6, 2, 1)]:
                b.set_schedule(ctas, stages, order)
                assert b.schedule() == (ctas, stages, order)
                for _ in range(2):  # two solves in a row
                    sw, h = b.solve(tol, 80)
                    np.testing.assert_array_equal(sw, sw0)
                    for k, (s, _, _) in enumerate(members):
                        np.testing.assert_array_equal(h[k], h0[k])
                        np.testing.assert_array_equal(s.solution(), u0[k])
        ctas, stages, order, ms = b.tune()
        assert ctas >= 1 and 2 <= stages <= 4 and order in (0, 1) and ms > 0
        assert b.schedule() == (ctas, stages, order) and b.warps_per_line() in (1, 2)
        sw, h = b.solve(tol, 80)
        np.testing.assert_array_equal(sw, sw0)
    finally:
        close_all(members, b)


@pytest.mark.parametrize("algo", [ALGO_FP64, ALGO_MIXED])
def test_batch_initial_and_refactor(algo):
    members = make_members(algo, pick={0, 1, 6})
    b = Batch([m[0] for m in members])
    try:
        tol = 1e-12 if algo == ALGO_FP64 else 1e-10
        s1, mesh1, _ = members[1]
        rng = np.random.default_rng(3)
        s1.set_initial(rng.uniform(-0.1, 0.1, 9 * mesh1.nelem))
        batch_vs_alone(members, b, tol, 80)
        s1.set_initial(None)
        # new values for member 2, same mesh and algorithm: the batch follows
        s2, mesh2, _ = members[2]
        s2.set_jacobian(Jacobian.generate(mesh2, 5.0, 11))
        s2.factor(algo)
        batch_vs_alone(members, b, tol, 80)
        # a new right-hand side for member 0
        s0, mesh0, _ = members[0]
        s0.set_rhs(rng.uniform(-1, 1, 9 * mesh0.nelem))
        batch_vs_alone(members, b, tol, 80)
    finally:
        close_all(members, b)


def test_batch_inner_schedule_equals_alone():
    members = make_members(ALGO_MIXED, pick={0, 1, 4, 6})
    for s, _, _ in members:
        s.set_inner_schedule(3, 5)
    b = Batch([m[0] for m in members])   # takes the first member's schedule
    try:
        batch_vs_alone(members, b, 1e-10, 80)
        b.set_inner_schedule(2, 4)
        for s, _, _ in members:
            s.set_inner_schedule(2, 4)
        batch_vs_alone(members, b, 1e-10, 80)
    finally:
        close_all(members, b)


def test_batch_sweep_limit_and_inner():
    members = make_members(ALGO_MIXED, pick={0, 4})
    b = Batch([m[0] for m in members])
    try:
        sw, h = b.solve(1e-30, 3)
        assert list(sw) == [3, 3] and all(len(x) == 4 for x in h)
        b.set_inner_sweeps(2)
        for s, _, _ in members:
            s.set_inner_sweeps(2)
        batch_vs_alone(members, b, 1e-10, 80)
    finally:
        close_all(members, b)


def test_batch_rejects_bad_members():
    members = make_members(ALGO_FP64, pick={0})
    other = make_members(ALGO_MIXED, pick={2})
    ref = make_members(ALGO_REFERENCE, pick={3})
    unfactored = Solver(0)
    unfactored.set_mesh(Mesh.structured(4, 4))
    try:
        with pytest.raises(TbsError):
            Batch([members[0][0], other[0][0]])       # two algorithms
        with pytest.raises(TbsError):
            Batch([ref[0][0]])                        # reference algorithm
        with pytest.raises(TbsError):
            Batch([unfactored])                       # not factored
        with pytest.raises(TbsError):
            Batch([members[0][0], members[0][0]])     # the same system twice
        b = Batch([members[0][0]])
        with pytest.raises(TbsError):
            b.set_schedule(1000, 2, 0)                # does not fit on an SM
        # re-factoring a member with another algorithm invalidates it in the batch
        members[0][0].factor(ALGO_MIXED)
        with pytest.raises(TbsError):
            b.solve(1e-10, 10)
        b.close()
    finally:
        close_all(members)
        close_all(other)
        close_all(ref)
        unfactored.close()
