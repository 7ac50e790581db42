"""Line partitions of one mesh on the GPU, through the C ABI.

Several partitions run in one process on one device, their halo lines'
updates copied between the contexts in stream order by the host (no kernel
waits for another).  Each partition sweeps with the TBS_ALGO_FP64 kernels,
so the owned cells' U is bit-identical to the FP64 sweep of the whole mesh
on the same GPU; the global norms are within 1e-12 of the initial residual
of that sweep and of the oracle's (the FP64 bar), and a solve to a
tolerance stops at the same sweep.
"""
import numpy as np
import pytest
import torch

import oracle
import triblocksolve_b200 as tbs
from meshes import ragged_mesh
from triblocksolve_b200 import _native as N
from triblocksolve_b200.partition import (LocalExchange, PartitionedSolve, PartitionSolver,
                                          gather_solution, partition_lines)

pytestmark = pytest.mark.gpu
TOL = 1e-12  # per sweep, relative to ||R_0||


def _problem(kind, shift=9.0, seed=3):
    mesh = tbs.Mesh.structured(*kind) if isinstance(kind, tuple) else \
        ragged_mesh([5, 9, 1, 7, 7, 3, 8, 2, 6, 9, 4, 12, 16, 1, 5], seed=seed)
    return mesh, tbs.Jacobian.generate(mesh, shift, seed)


def _whole(mesh, jac):
    s = tbs.Solver(0)
    s.set_mesh(mesh)
    s.set_jacobian(jac)
    s.factor(tbs.ALGO_FP64)
    return s


def _parts(mesh, jac, nparts):
    parts = partition_lines(mesh, nparts)
    sw = [PartitionSolver(p, 0) for p in parts]
    for p, s in zip(parts, sw):
        s.set_jacobian_arrays(*p.sub_arrays(jac.jacD, jac.jacO1, jac.jacO2, jac.rhs))
        s.factor(tbs.ALGO_FP64)
    return parts, sw


@pytest.mark.parametrize("kind,nparts", [((24, 32), 1), ((24, 32), 3), ("ragged", 4),
                                         ((60, 64), 7), ("ragged", 15), ((3, 40), 3)])
def test_partitions_match_the_whole_mesh(kind, nparts):
    mesh, jac = _problem(kind)
    n = 6
    whole = _whole(mesh, jac)
    hw = whole.sweep(n)
    Uw = whole.solution()
    ref = oracle.lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, n)
    parts, sw = _parts(mesh, jac, nparts)
    run = PartitionedSolve(sw, LocalExchange(parts, sw))
    hist = np.array([run.start()] + [run.sweep() for _ in range(n)])
    U = gather_solution(parts, [s.solution() for s in sw], mesh.nelem)
    assert np.array_equal(U, Uw)
    assert np.all(np.abs(hist - hw) <= TOL * hw[0])
    assert np.all(np.abs(hist - ref["hist"]) <= TOL * ref["hist"][0])
    # halo lines carry their owners' solution
    for p, s in zip(parts, sw):
        assert np.array_equal(s.solution().reshape(-1, 9), Uw.reshape(-1, 9)[p.elems])
    # the true residual over the owned cells adds up to the whole mesh's
    t = np.sqrt(sum(s.true_residual_norm() ** 2 for s in sw))
    tw = whole.true_residual_norm()
    assert abs(t - tw) <= 1e-12 * hw[0]
    whole.close()
    for s in sw:
        s.close()


def test_partitioned_solve_stops_at_the_same_sweep():
    mesh, jac = _problem((48, 40), shift=4.0)
    whole = _whole(mesh, jac)
    nw, hw = whole.solve(1e-10, 200)
    Uw = whole.solution()
    parts, sw = _parts(mesh, jac, 5)
    run = PartitionedSolve(sw, LocalExchange(parts, sw))
    n, hist = run.solve(1e-10, 200)
    assert n == nw
    assert np.all(np.abs(hist - hw) <= TOL * hw[0])
    assert np.array_equal(gather_solution(parts, [s.solution() for s in sw], mesh.nelem), Uw)
    # the convergence was checked against the true residual, as the whole mesh's was
    assert (run.checks, run.restarts) == (1, 0) and whole.solve_check()[1:] == (1, 0)
    true = np.sqrt(sum(s.true_residual_norm() ** 2 for s in sw))
    assert true <= 1e-10 * hist[0] * 1.0000001
    # a second solve of the same partitions repeats the first bit for bit
    n2, hist2 = run.solve(1e-10, 200)
    assert n2 == n and np.array_equal(hist2, hist)
    whole.close()
    for s in sw:
        s.close()


def test_partitioned_sweeps_restart_from_the_true_residual():
    """A check after every sweep: each check's true residual is the next
    line solves' input (tbs_part_solve_du forms it), so every sweep starts
    from rhs + J U as the reference's own sweep does; the checked norms
    follow the oracle's history and the solution the whole mesh's."""
    mesh, jac = _problem("ragged", shift=4.0)
    n = 5
    ref = oracle.lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, n)
    whole = _whole(mesh, jac)
    whole.sweep(n)
    Uw = whole.solution()
    parts, sw = _parts(mesh, jac, 4)
    run = PartitionedSolve(sw, LocalExchange(parts, sw))
    hist = [run.start()]
    for _ in range(n):
        run._solve_and_exchange()
        rec = float(run._line_res().item()) ** 0.5
        for s in sw:
            s.check_async()
        hist.append(float(run.ex.norm_sq_async(sw).item()) ** 0.5)
        assert abs(hist[-1] - rec) <= TOL * hist[0]
    hist = np.array(hist)
    assert np.all(np.abs(hist - ref["hist"]) <= TOL * ref["hist"][0])
    U = gather_solution(parts, [s.solution() for s in sw], mesh.nelem)
    assert np.max(np.abs(U - Uw)) <= 1e-12 * np.max(np.abs(Uw))
    # a check that ends the solve leaves the next start clean: a plain
    # partitioned sweep sequence afterwards repeats the first one's norms
    h2 = np.array([run.start()] + [run.sweep() for _ in range(n)])
    h1 = np.array([run.start()] + [run.sweep() for _ in range(n)])
    assert np.array_equal(h1, h2)
    whole.close()
    for s in sw:
        s.close()


def test_partition_refusals():
    mesh, jac = _problem((12, 16))
    parts, sw = _parts(mesh, jac, 2)
    s = sw[0]
    for call in (lambda: s.solve(1e-10, 10), lambda: s.sweep(1),
                 lambda: s.solve_multi(np.zeros((1, 9 * s.nelem)), 1e-10, 10),
                 lambda: s.gmres(1e-10, 5, 1, 10)):
        with pytest.raises(tbs.TbsError) as e:
            call()
        assert e.value.code == N.TBS_ERR_UNSUPPORTED
    s.factor(tbs.ALGO_REFERENCE)
    with pytest.raises(tbs.TbsError) as e:
        s.start()
    assert e.value.code == N.TBS_ERR_UNSUPPORTED
    buf = torch.zeros(9 * int(s.part.mesh.max_line_nelem), dtype=torch.float64, device="cuda")
    with pytest.raises(tbs.TbsError) as e:
        s.line_vector(N.VEC_UPDATE, 0, buf, False)
    assert e.value.code == N.TBS_ERR_UNSUPPORTED
    s.factor(tbs.ALGO_FP64)
    with pytest.raises(tbs.TbsError) as e:
        s.line_vector(N.VEC_UPDATE, s.part.mesh.nline, buf, False)
    assert e.value.code == N.TBS_ERR_ARG
    # owned lines' cells must come first
    rag = ragged_mesh([4, 6, 3, 5], seed=11)
    assert rag.lines[:rag.linepoint[rag.nline - 1]].max() >= rag.linepoint[rag.nline - 1]
    bad = tbs.Solver(0)
    with pytest.raises(tbs.TbsError) as e:
        N.check(N.lib.tbs_set_partition_mesh(bad.ctx, 1, rag.nvar, rag.nelem, rag.nintface,
                                             rag.eftot, rag.nline, rag.nlineelem, *rag._arrays()),
                bad.ctx)
    assert e.value.code == N.TBS_ERR_FORMAT
    bad.close()
    for x in sw:
        x.close()
