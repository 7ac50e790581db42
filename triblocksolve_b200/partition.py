"""Line partitions of one mesh: the LIJ sweep loop over several contexts.

The reference solves a mesh on one device (src/main.cxx:180-229).  A mesh
can also be split into contiguous ranges of lines, one per GPU (or several
on one GPU).  Lines are independent in the line solve
(linesmoothLU_TriBlock_v3.okl:92-226); the residual
(linesmoothLU_TriBlock_v3.okl:228-336) reads the update of the cells across
the cross-line faces, which may belong to another partition.  So each
partition's mesh holds its owned lines followed by *halo lines*: whole
copies of the other partitions' lines that hold a neighbour of an owned
cell.  One sweep is

    line solves of every line              (tbs_part_solve_du)
    halo lines' dU copied from their owners (the exchange, one message per
                                             neighbouring partition)
    residual, U += dU, norm of the owned   (tbs_part_line_res)
    global norm = sqrt(sum of the squares) (an all-reduce of one double)

The owned cells' U and dU are bit-identical to a sweep of the whole mesh
(the per-cell arithmetic does not change; only the global norm is summed
in another order).

``partition_lines`` builds the partitions (host-side index work, no GPU);
``PartitionSolver`` is one partition on a device (the C ABI); the exchanges
move the halo lines' vectors: ``LocalExchange`` between partitions of this
process, ``DistExchange`` between processes over ``torch.distributed``
(NCCL between GPUs, or gloo for host buffers).  ``PartitionedSolve`` runs
the sweep loop over either.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .lij import Mesh, Solver


@dataclass
class Partition:
    """One line range of a mesh and its halo lines.

    ``lines``: global line ids, the ``nowned`` owned lines then the halo
    lines (ascending).  ``elems`` / ``faces``: global element / face ids in
    the partition's local numbering (owned lines' cells first, in line
    order).  ``recvs[q]`` = local halo line indices whose update comes from
    partition q; ``sends[q]`` = local owned line indices partition q needs,
    in the same (ascending global id) order as q's ``recvs[self.index]``."""
    index: int
    lines: np.ndarray
    nowned: int
    elems: np.ndarray
    faces: np.ndarray
    mesh: Mesh
    nelem_own: int
    sends: dict = field(default_factory=dict)
    recvs: dict = field(default_factory=dict)

    @property
    def nhalo(self) -> int:
        return int(self.lines.size - self.nowned)

    def sub_arrays(self, jacD, jacO1, jacO2, rhs):
        """This partition's Jacobian arrays cut from the whole mesh's."""
        nv = self.mesh.nvar
        nb = nv * nv
        D = np.ascontiguousarray(np.asarray(jacD).reshape(-1, nb)[self.elems]).ravel()
        O1 = np.ascontiguousarray(np.asarray(jacO1).reshape(-1, nb)[self.faces]).ravel()
        O2 = np.ascontiguousarray(np.asarray(jacO2).reshape(-1, nb)[self.faces]).ravel()
        r = np.ascontiguousarray(np.asarray(rhs).reshape(-1, nv)[self.elems]).ravel()
        return D, O1, O2, r


def line_bounds(mesh: Mesh, nparts: int) -> np.ndarray:
    """First line of every partition (plus nline): contiguous ranges of about
    equal cell counts, each at least one line."""
    nline = int(mesh.nline)
    if nparts < 1 or nparts > nline:
        raise ValueError(f"cannot split {nline} lines into {nparts} partitions")
    cum = np.concatenate([[0], np.cumsum(np.asarray(mesh.linesize, np.int64))])
    total = cum[-1]
    b = [0]
    for p in range(1, nparts):
        target = total * p / nparts
        l = int(np.searchsorted(cum, target, side="left"))
        l = min(max(l, b[-1] + 1), nline - (nparts - p))
        b.append(l)
    b.append(nline)
    return np.array(b, np.int64)


def partition_lines(mesh: Mesh, nparts: int, bounds=None) -> list[Partition]:
    """Split ``mesh`` into ``nparts`` contiguous line ranges (``bounds``: the
    first line of each range plus nline, default ``line_bounds``)."""
    nv = int(mesh.nvar)
    ep, ef, fc = (np.asarray(getattr(mesh, f), np.int64) for f in ("epoint", "ef", "fc"))
    ls, lp, ln, lf = (np.asarray(getattr(mesh, f), np.int64)
                      for f in ("linesize", "linepoint", "lines", "lineface"))
    nline, nelem = int(mesh.nline), int(mesh.nelem)
    b = np.asarray(line_bounds(mesh, nparts) if bounds is None else bounds, np.int64)
    if b.size != nparts + 1 or b[0] != 0 or b[-1] != nline or np.any(np.diff(b) < 1):
        raise ValueError("bounds must rise from 0 to nline with at least one line per partition")
    line_of = np.empty(nelem, np.int64)
    line_of[ln] = np.repeat(np.arange(nline), ls)
    part_of_line = np.repeat(np.arange(nparts), np.diff(b))
    # every (element, face) entry of ef with the cell across the face
    ent_e = np.repeat(np.arange(nelem), np.diff(ep))
    ent_f = ef.copy()
    inner = ent_f >= 0
    fi = np.where(inner, ent_f, 0)
    ent_nb = np.where(fc[2 * fi] == ent_e, fc[2 * fi + 1], fc[2 * fi])
    ent_part = part_of_line[line_of[ent_e]]
    nb_part = np.where(inner, part_of_line[line_of[ent_nb]], -1)

    def ranges(first, count):
        """concatenated index ranges first[i] .. first[i] + count[i] - 1"""
        count = np.asarray(count, np.int64)
        off = np.repeat(np.asarray(first, np.int64) - np.concatenate([[0], np.cumsum(count)[:-1]]),
                        count)
        return off + np.arange(int(count.sum()))

    parts = []
    for p in range(nparts):
        owned = np.arange(b[p], b[p + 1])
        sel = inner & (ent_part == p) & (nb_part != p)
        halo = np.unique(line_of[ent_nb[sel]])
        lines = np.concatenate([owned, halo]).astype(np.int64)
        elems = ln[ranges(lp[lines], ls[lines])]
        nelem_own = int(ls[owned].sum())
        g2l = np.full(nelem, -1, np.int64)
        g2l[elems] = np.arange(elems.size)
        # faces with both cells in this partition's mesh, in global order
        ent = ranges(ep[elems], ep[elems + 1] - ep[elems])  # ef entries of the local cells
        f_in = ent_f[ent]
        both = (f_in >= 0)
        fb = np.where(both, f_in, 0)
        both &= (g2l[fc[2 * fb]] >= 0) & (g2l[fc[2 * fb + 1]] >= 0)
        faces = np.unique(f_in[both])
        f2l = np.full(max(int(mesh.nintface), 1), -1, np.int64)
        f2l[faces] = np.arange(faces.size)
        # element-face lists in the original order; dropped faces become -1
        sub_ef = np.where(f_in < 0, f_in, f2l[np.where(f_in >= 0, f_in, 0)])
        sub_ep = np.concatenate([[0], np.cumsum(ep[elems + 1] - ep[elems])])
        sub_fc = np.stack([g2l[fc[2 * faces]], g2l[fc[2 * faces + 1]]], axis=1).ravel()
        sub_ls = ls[lines]
        sub_lp = np.concatenate([[0], np.cumsum(sub_ls)])
        lf_in = lf[ranges(lp[lines], ls[lines])]
        sub_lf = np.where(lf_in >= 0, f2l[np.where(lf_in >= 0, lf_in, 0)], -1)
        sub = Mesh.from_arrays(nv, epoint=sub_ep, ef=sub_ef, fc=sub_fc, linesize=sub_ls,
                               linepoint=sub_lp, lines=np.arange(elems.size), lineface=sub_lf)
        parts.append(Partition(index=p, lines=lines, nowned=int(owned.size), elems=elems,
                               faces=faces, mesh=sub, nelem_own=nelem_own))
    # who sends which lines to whom (ascending global line id on both sides)
    for p, part in enumerate(parts):
        for k in range(part.nowned, part.lines.size):
            g = int(part.lines[k])
            q = int(part_of_line[g])
            part.recvs.setdefault(q, []).append(k)
            parts[q].sends.setdefault(p, []).append(int(g - b[q]))
    return parts


def gather_solution(parts: list[Partition], local_U: list[np.ndarray], nelem: int) -> np.ndarray:
    """The whole mesh's U (element order) from every partition's owned rows."""
    nv = parts[0].mesh.nvar
    U = np.zeros(nv * nelem)
    for part, u in zip(parts, local_U):
        rows = np.asarray(u).reshape(-1, nv)[:part.nelem_own]
        U.reshape(-1, nv)[part.elems[:part.nelem_own]] = rows
    return U


class PartitionSolver(Solver):
    """One partition on a device: ``tbs_set_partition_mesh`` and the split
    sweep (TBS_ALGO_FP64, nvar 9)."""

    def __init__(self, part: Partition, device_id: int = 0):
        super().__init__(device_id)
        self.part = part
        m = part.mesh
        self._chk(N.lib.tbs_set_partition_mesh(self.ctx, part.nhalo, m.nvar, m.nelem, m.nintface,
                                               m.eftot, m.nline, m.nlineelem, *m._arrays()))
        self.nvar, self.nelem = m.nvar, m.nelem

    def start(self) -> float:
        n = C.c_double()
        self._chk(N.lib.tbs_part_start(self.ctx, C.byref(n)))
        return n.value

    def solve_du(self) -> None:
        self._chk(N.lib.tbs_part_solve_du(self.ctx))

    def line_res(self) -> float:
        n = C.c_double()
        self._chk(N.lib.tbs_part_line_res(self.ctx, C.byref(n)))
        return n.value

    def line_res_async(self) -> None:
        """tbs_part_line_res without reading the norm (no host synchronisation)."""
        self._chk(N.lib.tbs_part_line_res(self.ctx, None))

    def check_async(self) -> None:
        """tbs_part_check without reading the norm: the true residual of the
        owned cells (the next solve_du forms its input from it)."""
        self._chk(N.lib.tbs_part_check(self.ctx, None))

    def owned_norm_to(self, t) -> None:
        """The owned norm into the one-element tensor ``t``, in stream order."""
        self._chk(N.lib.tbs_part_owned_norm(self.ctx, C.c_void_p(t.data_ptr())))

    def sync(self) -> None:
        self._chk(N.lib.tbs_sync(self.ctx))

    def lines_vector(self, which: int, lines, buf, to_line: bool) -> None:
        """Several lines' vectors packed back to back into ``buf`` (or
        unpacked from it) by one launch."""
        ls = np.ascontiguousarray(lines, np.int32)
        ptr = buf if isinstance(buf, int) else buf.data_ptr()
        self._chk(N.lib.tbs_part_lines_vector(self.ctx, which, int(ls.size), N.iptr(ls),
                                              C.c_void_p(ptr), 1 if to_line else 0))

    def line_vector(self, which: int, line: int, buf, to_line: bool) -> None:
        """Copy a line's vector to / from ``buf`` (a CUDA tensor of
        linesize * 9 doubles, or its address)."""
        ptr = buf if isinstance(buf, int) else buf.data_ptr()
        self._chk(N.lib.tbs_part_line_vector(self.ctx, which, line, C.c_void_p(ptr),
                                             1 if to_line else 0))


def _line_len(part: Partition, k: int) -> int:
    return int(part.mesh.linesize[k]) * int(part.mesh.nvar)


class LocalExchange:
    """Halo exchange between partitions that live in this process on one
    device: each halo line's vector is copied from its owner into the
    receiver through a staging buffer, in the order of one stream.  (Across
    devices or processes use ``DistExchange``.)"""

    def __init__(self, parts: list[Partition], sweepers: list, device: str = "cuda"):
        import torch
        self.parts, self.sweepers = parts, sweepers
        dev = torch.device(device)
        if dev.type == "cuda":
            want = dev.index if dev.index is not None else torch.cuda.current_device()
            for s in sweepers:
                got = getattr(getattr(s, "platform", None), "device_id", want)
                if got != want:
                    raise ValueError(f"LocalExchange: a partition is on device {got}, the "
                                     f"exchange on device {want}; use DistExchange across devices")
        longest = max(int(p.mesh.max_line_nelem) for p in parts) * int(parts[0].mesh.nvar)
        self.buf = torch.empty(longest, dtype=torch.float64, device=device)
        if self.buf.is_cuda:
            # one stream for every partition: each copy then follows the
            # owner's line solves and precedes the receiver's residual
            self.stream = torch.cuda.current_stream(self.buf.device)
            for s in sweepers:
                s.set_stream(self.stream.cuda_stream)

    def exchange(self, which: int) -> None:
        for p, part in enumerate(self.parts):
            for q, ks in part.recvs.items():
                src = self.parts[q].sends[p]
                for k_dst, k_src in zip(ks, src):
                    n = _line_len(part, k_dst)
                    self.sweepers[q].line_vector(which, k_src, self.buf[:n], False)
                    self.sweepers[p].line_vector(which, k_dst, self.buf[:n], True)

    def allreduce_sum(self, x: float) -> float:
        return x

    def norm_sq_async(self, sweepers):
        """Sum of the squared owned norms as a one-element tensor, not yet read."""
        return owned_norm_sq(sweepers, self.buf.device)


def owned_norm_sq(sweepers, device):
    """Sum of the sweepers' squared owned norms as a one-element tensor on
    `device`, formed in stream order without a host read."""
    import torch
    t = torch.zeros(1, dtype=torch.float64, device=device)
    one = torch.empty(1, dtype=torch.float64, device=device)
    for s in sweepers:
        s.owned_norm_to(one)
        t.addcmul_(one, one)
    return t


class DistExchange:
    """Halo exchange of this process's partition with the others over
    ``torch.distributed`` (the process group's backend: NCCL for CUDA
    buffers, gloo for host buffers): one message per neighbouring
    partition and direction, posted together."""

    def __init__(self, part: Partition, sweeper, device="cuda", group=None):
        import torch
        import torch.distributed as dist
        self.torch, self.dist, self.group = torch, dist, group
        self.part, self.sweeper, self.device = part, sweeper, device
        self.sendbufs, self.recvbufs = {}, {}
        if torch.device(device).type == "cuda":
            # the context launches on torch's current stream, which the
            # process group's sends and receives are ordered against
            sweeper.set_stream(torch.cuda.current_stream(torch.device(device)).cuda_stream)
        for q, ks in sorted(part.sends.items()):
            n = sum(_line_len(part, k) for k in ks)
            self.sendbufs[q] = torch.empty(n, dtype=torch.float64, device=device)
        for q, ks in sorted(part.recvs.items()):
            n = sum(_line_len(part, k) for k in ks)
            self.recvbufs[q] = torch.empty(n, dtype=torch.float64, device=device)

    def _lines(self, buf, ks):
        off = 0
        for k in ks:
            n = _line_len(self.part, k)
            yield k, buf[off:off + n]
            off += n

    def exchange(self, which: int) -> None:
        # one pack launch per neighbour and direction
        for q, ks in sorted(self.part.sends.items()):
            self.sweeper.lines_vector(which, ks, self.sendbufs[q], False)
        ops = [self.dist.P2POp(self.dist.isend, self.sendbufs[q], q, self.group)
               for q in sorted(self.sendbufs)]
        ops += [self.dist.P2POp(self.dist.irecv, self.recvbufs[q], q, self.group)
                for q in sorted(self.recvbufs)]
        if ops:
            for w in self.dist.batch_isend_irecv(ops):
                w.wait()
        for q, ks in sorted(self.part.recvs.items()):
            self.sweeper.lines_vector(which, ks, self.recvbufs[q], True)

    def allreduce_sum(self, x: float) -> float:
        t = self.torch.tensor([x], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, group=self.group)
        return float(t.item())

    def norm_sq_async(self, sweepers):
        """The global sum of the squared owned norms as a one-element tensor:
        the owned norms copied on the device, squared and all-reduced in
        stream order, not yet read by the host."""
        t = owned_norm_sq(sweepers, self.torch.device(self.device))
        self.dist.all_reduce(t, group=self.group)
        return t


class PartitionedSolve:
    """The sweep loop of src/main.cxx:207-229 over line partitions: the
    sweepers of this process (one per partition it holds) and an exchange
    (``LocalExchange`` or ``DistExchange``).  The convergence test is the
    one of ``tbs_solve`` on the global norm."""

    def __init__(self, sweepers: list, exchange, check: bool = True):
        self.sweepers, self.ex = sweepers, exchange
        self.check = check  # the true-residual check at convergence, as tbs_solve's
        self.checks = self.restarts = 0

    def _global(self, norms) -> float:
        return math.sqrt(self.ex.allreduce_sum(sum(n * n for n in norms)))

    def start(self) -> float:
        return self._global([s.start() for s in self.sweepers])

    def sweep(self) -> float:
        for s in self.sweepers:
            s.solve_du()
        self.ex.exchange(N.VEC_UPDATE)
        return self._global([s.line_res() for s in self.sweepers])

    def _solve_and_exchange(self) -> None:
        for s in self.sweepers:
            s.solve_du()
        self.ex.exchange(N.VEC_UPDATE)

    def _line_res(self):
        for s in self.sweepers:
            s.line_res_async()
        return self.ex.norm_sq_async(self.sweepers)

    def solve(self, rel_tol: float, max_sweeps: int = 1000):
        """Sweeps from U = 0 until ||R|| <= rel_tol ||R_0|| or max_sweeps;
        returns (sweeps, global norm history).

        One host read per sweep: the owned norms stay on the device, are
        squared and all-reduced there, and the host reads the global norm
        only after it has issued the next sweep's line solves and halo
        exchange, which therefore overlap the read and the convergence
        test.  When the test ends the solve, that speculative line solve
        is discarded: U and the norms are those of the last sweep counted;
        the context's last update (tbs_get_update) is the discarded one.
        Every rank takes the same decisions from the same global norm, so
        the collectives stay matched.

        When the recursive norm meets the tolerance, the true residual
        rhs + J U is formed from the original blocks (tbs_part_check) and
        its global norm decides: at or below the tolerance the solve ends
        with the history unchanged; above it, that norm replaces the last
        entry and the sweeps go on from the true residual."""
        n0 = self.start()
        hist = [n0]
        self.checks = self.restarts = 0
        go = lambda g: math.isfinite(g) and g > rel_tol * n0
        if max_sweeps < 1 or not go(n0):
            return 0, np.array(hist)
        self._solve_and_exchange()
        pending = self._line_res()
        while True:
            more = len(hist) < max_sweeps  # a sweep after the one being read is allowed
            if more:
                self._solve_and_exchange()
            g = math.sqrt(float(pending.item()))
            hist.append(g)
            if go(g):
                if not more:
                    break
                pending = self._line_res()
                continue
            if not (self.check and math.isfinite(g)):
                break
            for s in self.sweepers:
                s.check_async()
            t = math.sqrt(float(self.ex.norm_sq_async(self.sweepers).item()))
            self.checks += 1
            if t <= rel_tol * n0:
                break
            if not math.isfinite(t):
                hist[-1] = t
                break
            self.restarts += 1
            hist[-1] = t
            if not more:
                break
            self._solve_and_exchange()  # from the true residual: the speculative one is stale
            pending = self._line_res()
        for s in self.sweepers:
            s.sync()
        return len(hist) - 1, np.array(hist)
