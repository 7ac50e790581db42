"""Line partitions of one mesh, on the CPU (no GPU).

The partitioner and both halo exchanges are host logic; here each
partition is swept by the oracle (the reference's own line solve and
residual rule, oracle/lij_oracle.c) instead of the GPU kernels, so that the
partitioned sweep loop is checked against the oracle's sweep of the whole
mesh: the owned cells' U bit-identical, the global norms within rounding of
the summation order.  The exchange over torch.distributed runs as gloo
ranks (world sizes 2 and 3: a middle partition has two neighbours).
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import oracle
import triblocksolve_b200 as tbs
from meshes import ragged_mesh
from triblocksolve_b200.partition import (DistExchange, LocalExchange, PartitionedSolve,
                                          gather_solution, line_bounds, partition_lines)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NORM_TOL = 1e-13  # relative to ||R_0||: the global norm sums the partitions' squares


class OracleSweeper:
    """One partition swept by the oracle, with PartitionSolver's interface.
    Vectors are element-ordered numpy arrays; a line's vector travels in
    the line's cell order."""

    def __init__(self, part, jacD, jacO1, jacO2, rhs):
        self.part = part
        m = part.mesh
        self.nv = int(m.nvar)
        self.D, self.O1, self.O2, self.rhs = part.sub_arrays(jacD, jacO1, jacO2, rhs)
        self.base = oracle.Baseline(m, self.D, self.O1, self.O2, self.rhs, 1)
        self.own = part.nelem_own * self.nv

    def _ptrs(self):
        ip = lambda f: self.base._ints[f].ctypes.data_as(oracle._ip)
        return ip

    def _norm(self):
        r = self.base.R[:self.own]
        return float(np.sqrt(np.dot(r, r)))

    def start(self):
        self.base.reset()
        return self._norm()

    def solve_du(self):
        b, ip = self.base, self._ptrs()
        oracle.lib.oracle_solve_du(self.nv, b.nline, ip("linesize"), ip("linepoint"), ip("lines"),
                                   oracle._dp_(b.DLU), oracle._dp_(b.DinvC), oracle._dp_(b.A),
                                   oracle._dp_(b.dU), oracle._dp_(b.R))

    def line_res(self):
        b, ip = self.base, self._ptrs()
        b.U += b.dU
        b.R[:] = self.rhs
        oracle.lib.oracle_line_res(self.nv, b.nline, ip("epoint"), ip("ef"), ip("fc"), ip("linesize"),
                                   ip("linepoint"), ip("lines"), oracle._dp_(self.D),
                                   oracle._dp_(self.O1), oracle._dp_(self.O2), oracle._dp_(b.U),
                                   oracle._dp_(b.R))
        return self._norm()

    def line_res_async(self):
        self.line_res()

    def check_async(self):
        pass  # the oracle's R is the true residual already

    def owned_norm_to(self, t):
        t[0] = self._norm()

    def sync(self):
        pass

    def lines_vector(self, which, ks, buf, to_line):
        off = 0
        for k in ks:
            n = int(self.part.mesh.linesize[k]) * self.nv
            self.line_vector(which, k, buf[off:off + n], to_line)
            off += n

    def line_vector(self, which, k, buf, to_line):
        m = self.part.mesh
        cells = m.lines[m.linepoint[k]:m.linepoint[k] + m.linesize[k]]
        vec = (self.base.U if which == tbs._native.VEC_SOLUTION else self.base.dU).reshape(-1, self.nv)
        if to_line:
            vec[cells] = buf.numpy().reshape(-1, self.nv)
        else:
            buf.copy_(torch.from_numpy(vec[cells].ravel()))


def _problem(lens, seed, shift=9.0):
    mesh = ragged_mesh(lens, seed=seed)
    jac = tbs.Jacobian.generate(mesh, shift, seed + 1)
    return mesh, jac


LENS = [5, 9, 1, 7, 7, 3, 8, 2, 6, 9, 4]


def test_partition_maps_cover_the_mesh():
    mesh, _ = _problem(LENS, 3)
    for nparts in (1, 2, 3, 5, len(LENS)):
        parts = partition_lines(mesh, nparts)
        owned = np.concatenate([p.elems[:p.nelem_own] for p in parts])
        assert np.array_equal(np.sort(owned), np.arange(mesh.nelem))
        for p in parts:
            p.mesh.validate()
            assert p.mesh.nelem == p.elems.size and p.mesh.nintface == p.faces.size
            # every face of an owned cell is in the partition's mesh
            own = set(p.elems[:p.nelem_own].tolist())
            inside = set(p.elems.tolist())
            for e in own:
                for f in mesh.ef[mesh.epoint[e]:mesh.epoint[e + 1]]:
                    if f >= 0:
                        assert int(f) in set(p.faces.tolist())
                        assert int(mesh.fc[2 * f]) in inside and int(mesh.fc[2 * f + 1]) in inside
            # what p receives from q is what q sends to p, line for line
            for q, ks in p.recvs.items():
                src = parts[q].sends[p.index]
                assert [int(p.lines[k]) for k in ks] == [int(parts[q].lines[k]) for k in src]
                assert all(k < parts[q].nowned for k in src) and all(k >= p.nowned for k in ks)
        if nparts == 1:
            assert parts[0].nhalo == 0 and not parts[0].sends


def test_line_bounds_balance_cells():
    mesh, _ = _problem(LENS, 4)
    b = line_bounds(mesh, 3)
    assert b[0] == 0 and b[-1] == mesh.nline and np.all(np.diff(b) >= 1)
    with pytest.raises(ValueError):
        line_bounds(mesh, mesh.nline + 1)


@pytest.mark.parametrize("nparts", [1, 2, 4])
def test_local_partitions_match_whole_mesh_oracle(nparts):
    mesh, jac = _problem(LENS, 5)
    iters = 6
    ref = oracle.lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, iters)
    parts = partition_lines(mesh, nparts)
    sw = [OracleSweeper(p, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs) for p in parts]
    run = PartitionedSolve(sw, LocalExchange(parts, sw, device="cpu"))
    hist = [run.start()] + [run.sweep() for _ in range(iters)]
    assert np.all(np.abs(np.array(hist) - ref["hist"]) <= NORM_TOL * ref["hist"][0])
    U = gather_solution(parts, [s.base.U for s in sw], mesh.nelem)
    assert np.array_equal(U, ref["U"])
    # a halo line's U is its owner's
    for p, s in zip(parts, sw):
        rows = s.base.U.reshape(-1, 9)
        assert np.array_equal(rows, ref["U"].reshape(-1, 9)[p.elems])


def test_local_partitioned_solve_stops_like_the_whole_mesh():
    mesh, jac = _problem(LENS, 6)
    ref = oracle.lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, 40)
    tol = 1e-10
    want = int(np.argmax(ref["hist"] <= tol * ref["hist"][0]))
    parts = partition_lines(mesh, 3)
    sw = [OracleSweeper(p, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs) for p in parts]
    n, hist = PartitionedSolve(sw, LocalExchange(parts, sw, device="cpu")).solve(tol, 40)
    assert n == want
    assert np.all(np.abs(hist - ref["hist"][:n + 1]) <= NORM_TOL * ref["hist"][0])


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, port, out, world=2):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        mesh, jac = _problem(LENS, 7)
        parts = partition_lines(mesh, world)
        part = parts[rank]
        s = OracleSweeper(part, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs)
        run = PartitionedSolve([s], DistExchange(part, s, device="cpu"))
        n, hist = run.solve(1e-12, 30)
        out[rank] = (n, hist.tolist(), s.base.U[:part.nelem_own * 9].tolist(),
                     part.elems[:part.nelem_own].tolist())
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_match_whole_mesh_oracle(world):
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(port, out, world), nprocs=world, join=True)
        res = dict(out)
    mesh, jac = _problem(LENS, 7)
    ref = oracle.lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, 30)
    want = int(np.argmax(ref["hist"] <= 1e-12 * ref["hist"][0]))
    U = np.zeros(9 * mesh.nelem)
    for rank in range(world):
        n, hist, u, elems = res[rank]
        assert n == want
        assert np.all(np.abs(np.array(hist) - ref["hist"][:n + 1]) <= NORM_TOL * ref["hist"][0])
        U.reshape(-1, 9)[elems] = np.array(u).reshape(-1, 9)
    # every rank stopped at the same sweep: the whole-mesh U after `want` sweeps
    ref_n = oracle.lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, want)
    assert np.array_equal(U, ref_n["U"])


@pytest.mark.parametrize("world", [2, 3])
def test_torchrun_ranks_match_whole_mesh_oracle(world, tmp_path):
    """The partitioned solve as separate processes launched by torchrun (the
    launch and environment contract of bench.py --gpus N) on gloo: every
    rank stops at the whole mesh's sweep count and the owned cells' U is
    bit-identical to the oracle's whole-mesh sweep."""
    import subprocess
    lens, seed, tol = [6, 2, 9, 4, 8, 1, 7, 5], 9, 1e-11
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={world}", "--master-addr=127.0.0.1",
           f"--master-port={_free_port()}",
           os.path.join(ROOT, "tests", "partition_rank_worker.py"), str(tmp_path),
           ",".join(map(str, lens)), str(seed), repr(tol)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, OMP_NUM_THREADS="1"))
    assert r.returncode == 0, r.stderr[-3000:]
    mesh, jac = _problem(lens, seed)
    ref = oracle.lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, 40)
    want = int(np.argmax(ref["hist"] <= tol * ref["hist"][0]))
    U = np.zeros(9 * mesh.nelem)
    for rank in range(world):
        d = np.load(os.path.join(tmp_path, f"rank{rank}.npz"))
        assert int(d["n"]) == want
        assert np.all(np.abs(d["hist"] - ref["hist"][:want + 1]) <= NORM_TOL * ref["hist"][0])
        U.reshape(-1, 9)[d["elems"]] = d["U"].reshape(-1, 9)
    np.testing.assert_array_equal(U, oracle.lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs,
                                                want)["U"])


@pytest.mark.parametrize("limit", [1, 3])
def test_partitioned_solve_sweep_limit_discards_the_speculative_sweep(limit):
    """The loop issues the next sweep's line solves before it reads the
    global norm; at the sweep limit (and at convergence) that line solve is
    discarded: U is the whole mesh's after exactly `limit` sweeps."""
    mesh, jac = _problem(LENS, 11)
    parts = partition_lines(mesh, 3)
    sw = [OracleSweeper(p, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs) for p in parts]
    n, hist = PartitionedSolve(sw, LocalExchange(parts, sw, device="cpu")).solve(1e-30, limit)
    assert n == limit and hist.size == limit + 1
    ref = oracle.lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, limit)
    np.testing.assert_array_equal(gather_solution(parts, [s.base.U for s in sw], mesh.nelem),
                                  ref["U"])
    assert np.all(np.abs(hist - ref["hist"]) <= NORM_TOL * ref["hist"][0])
