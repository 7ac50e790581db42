"""The request loop (tbs_server_*) on the GPU.

Stated tolerance: none needed -- every right-hand side's solution, sweep
count and relative residual must be bit-identical to Solver.solve of the same
system and right-hand side alone, whether the request ran alone on the server
or in a mix of concurrent requests of other systems, sizes and right-hand-side
counts (continuous batching), with and without re-factorizations, under a
device budget that forces requests to queue.
"""
import threading

import numpy as np
import pytest

from meshes import ragged_mesh
from triblocksolve_b200 import ALGO_FP64, ALGO_MIXED, Jacobian, Mesh, Server, Solver
from triblocksolve_b200._native import TbsError

pytestmark = pytest.mark.gpu

SHAPES = [
    (lambda: Mesh.structured(20, 24), 9.0, 1),
    (lambda: ragged_mesh([5, 1, 7, 3, 3, 8, 13, 2, 9], seed=4), 9.0, 2),
    (lambda: Mesh.structured(48, 64), 6.0, 3),
    (lambda: Mesh.structured(1, 37), 9.0, 4),
]
TOL = 1e-10


def systems():
    out = []
    for mk, shift, seed in SHAPES:
        mesh = mk()
        out.append((mesh, Jacobian.generate(mesh, shift, seed)))
    return out


def alone(mesh, jac, rhs_rows, algo, tol=TOL, max_sweeps=200):
    """Reference results: a plain context per right-hand side."""
    s = Solver(0)
    try:
        s.set_mesh(mesh)
        s.set_jacobian(jac)
        s.factor(algo)
        res = []
        for r in rhs_rows:
            s.set_rhs(r)
            n, h = s.solve(tol, max_sweeps)
            res.append((s.solution(), n, h[-1] / h[0] if h[0] > 0 else 0.0))
        return res
    finally:
        s.close()


def check(req_result, expected):
    U, sw, rel, lat, q = req_result
    assert lat >= q >= 0.0
    for k, (u, n, r) in enumerate(expected):
        assert sw[k] == n
        np.testing.assert_array_equal(U[k], u)
        assert rel[k] == r
        assert r <= TOL


@pytest.mark.parametrize("algo", [ALGO_FP64, ALGO_MIXED])
def test_same_alone_and_in_the_mix(algo):
    sy = systems()
    rng = np.random.default_rng(7)
    # FP64: two lanes (the 48x64 system sweeps apart from the small ones)
    srv = Server(0, algo, budget_bytes=8 << 30, max_rhs=32, chunk=2,
                 lane_split=1000 if algo == ALGO_FP64 else 0)
    try:
        ids = [srv.add_system(m, j) for m, j in sy]
        probe_sys = 2
        probe_rhs = rng.uniform(-1, 1, (3, 9 * sy[probe_sys][0].nelem))
        expected = alone(*sy[probe_sys], probe_rhs, algo)
        # alone on the server
        check(srv.submit(ids[probe_sys], probe_rhs, TOL).wait(), expected)
        # in a mix: many requests in flight, the probe submitted in the middle
        mix = []
        for k in range(14):
            s = int(rng.integers(len(sy)))
            rows = rng.uniform(-1, 1, (int(rng.integers(1, 5)), 9 * sy[s][0].nelem))
            mix.append((s, rows, srv.submit(ids[s], rows, TOL)))
            if k == 6:
                probe = srv.submit(ids[probe_sys], probe_rhs, TOL)
        check(probe.wait(), expected)
        for s, rows, req in mix:
            check(req.wait(), alone(*sy[s], rows, algo))
        st = srv.stats()
        assert st["requests_done"] == 16 and st["peak_rhs_in_flight"] > 4
        assert st["graph_launches"] > 1
    finally:
        srv.close()


def test_refactor_requests_and_order():
    sy = systems()
    rng = np.random.default_rng(3)
    srv = Server(0, ALGO_FP64, budget_bytes=8 << 30, max_rhs=16, chunk=3)
    try:
        ids = [srv.add_system(m, j) for m, j in sy]
        mesh, jac = sy[0]
        new_jac = Jacobian.generate(mesh, 5.0, 99)
        r1 = rng.uniform(-1, 1, (2, 9 * mesh.nelem))
        r2 = rng.uniform(-1, 1, (1, 9 * mesh.nelem))
        r3 = rng.uniform(-1, 1, (1, 9 * mesh.nelem))
        other = rng.uniform(-1, 1, (2, 9 * sy[2][0].nelem))
        a = srv.submit(ids[0], r1, TOL)                        # old factors
        b = srv.submit(ids[0], r2, TOL, new_jacobian=new_jac)  # waits for a, re-factors
        o = srv.submit(ids[2], other, TOL)                     # not held back by the re-factor
        c = srv.submit(ids[0], r3, TOL)                        # new factors
        check(a.wait(), alone(mesh, jac, r1, ALGO_FP64))
        check(b.wait(), alone(mesh, new_jac, r2, ALGO_FP64))
        check(c.wait(), alone(mesh, new_jac, r3, ALGO_FP64))
        check(o.wait(), alone(*sy[2], other, ALGO_FP64))
        assert srv.stats()["refactors"] == 1
    finally:
        srv.close()


def test_admission_by_footprint():
    sy = systems()
    rng = np.random.default_rng(5)
    probe = Server(0, ALGO_FP64, budget_bytes=8 << 30, max_rhs=64)
    sid = probe.add_system(*sy[2])
    resident, per_rhs = probe.system_bytes(sid, 200)
    probe.close()
    # room for the system and two right-hand sides: requests of two queue up
    srv = Server(0, ALGO_FP64, budget_bytes=resident + 2 * per_rhs + per_rhs // 2, max_rhs=64)
    try:
        sid = srv.add_system(*sy[2])
        reqs = []
        for _ in range(6):
            rows = rng.uniform(-1, 1, (2, 9 * sy[2][0].nelem))
            reqs.append((rows, srv.submit(sid, rows, TOL)))
        with pytest.raises(TbsError):
            srv.submit(sid, rng.uniform(-1, 1, (3, 9 * sy[2][0].nelem)), TOL)  # never fits
        for rows, r in reqs:
            check(r.wait(), alone(*sy[2], rows, ALGO_FP64))
        st = srv.stats()
        assert st["peak_rhs_in_flight"] == 2
        assert st["peak_rhs_bytes"] <= 2 * per_rhs
    finally:
        srv.close()


def test_many_members_of_one_system_same_as_alone():
    """Twelve right-hand sides of one system in flight at once (the engine
    runs them as groups of 8 and 4 in the multi-RHS line solve and together
    in the grouped residual) beside another system's: each equals its solve
    alone."""
    sy = systems()
    rng = np.random.default_rng(21)
    srv = Server(0, ALGO_FP64, budget_bytes=8 << 30, max_rhs=32, chunk=3, lane_split=0)
    try:
        ids = [srv.add_system(m, j) for m, j in sy]
        big, other = 2, 0
        reqs = []
        for k in range(3):
            rows = rng.uniform(-1, 1, (4, 9 * sy[big][0].nelem))
            reqs.append((big, rows, srv.submit(ids[big], rows, TOL)))
            rows2 = rng.uniform(-1, 1, (1, 9 * sy[other][0].nelem))
            reqs.append((other, rows2, srv.submit(ids[other], rows2, TOL)))
        for s, rows, r in reqs:
            check(r.wait(), alone(*sy[s], rows, ALGO_FP64))
    finally:
        srv.close()


def test_three_lanes_same_as_alone():
    """Lane splits [100, 1000]: the 51- and 37-cell systems sweep in lane 0,
    the 480-cell one in lane 1, the 3,072-cell one in lane 2."""
    sy = systems()
    rng = np.random.default_rng(13)
    srv = Server(0, ALGO_FP64, budget_bytes=8 << 30, max_rhs=32, chunk=2, lane_split=[100, 1000])
    try:
        ids = [srv.add_system(m, j) for m, j in sy]
        reqs = []
        for k in range(12):
            s = k % len(sy)
            rows = rng.uniform(-1, 1, (int(rng.integers(1, 4)), 9 * sy[s][0].nelem))
            reqs.append((s, rows, srv.submit(ids[s], rows, TOL)))
        for s, rows, r in reqs:
            check(r.wait(), alone(*sy[s], rows, ALGO_FP64))
    finally:
        srv.close()
    with pytest.raises(TbsError):
        Server(0, ALGO_FP64, budget_bytes=1 << 30, lane_split=[1000, 100])   # not ascending
    with pytest.raises(TbsError):
        Server(0, ALGO_FP64, budget_bytes=1 << 30, lane_split=[1, 2, 3, 4])  # too many


def test_concurrent_clients():
    sy = systems()
    srv = Server(0, ALGO_FP64, budget_bytes=8 << 30, max_rhs=32, chunk=1, lane_split=500)
    try:
        ids = [srv.add_system(m, j) for m, j in sy]
        results, errors = {}, []

        def client(seed):
            try:
                rng = np.random.default_rng(seed)
                mine = []
                for _ in range(5):
                    s = int(rng.integers(len(sy)))
                    rows = rng.uniform(-1, 1, (int(rng.integers(1, 4)), 9 * sy[s][0].nelem))
                    mine.append((s, rows, srv.submit(ids[s], rows, TOL)))
                results[seed] = [(s, rows, r.wait()) for s, rows, r in mine]
            except Exception as ex:  # surfaced below
                errors.append(ex)

        th = [threading.Thread(target=client, args=(k,)) for k in range(4)]
        for t in th:
            t.start()
        for t in th:
            t.join(timeout=120)
        assert not errors, errors
        assert len(results) == 4
        for seed, lst in results.items():
            for s, rows, res in lst:
                check(res, alone(*sy[s], rows, ALGO_FP64))
    finally:
        srv.close()


def test_bad_requests():
    sy = systems()
    srv = Server(0, ALGO_FP64, budget_bytes=4 << 30, max_rhs=4)
    try:
        sid = srv.add_system(*sy[0])
        n = 9 * sy[0][0].nelem
        with pytest.raises(TbsError):
            srv.submit(sid + 5, np.zeros(n), TOL)             # unknown system
        with pytest.raises(TbsError):
            srv.submit(sid, np.zeros((5, n)), TOL)            # more right-hand sides than slots
        # a zero right-hand side is done at once with zero sweeps
        U, sw, rel, _, _ = srv.submit(sid, np.zeros(n), TOL).wait()
        assert sw[0] == 0 and rel[0] == 0.0 and not U.any()
    finally:
        srv.close()
    with pytest.raises(TbsError):
        Server(0, 0, budget_bytes=1 << 30)                     # reference algorithm: no server
