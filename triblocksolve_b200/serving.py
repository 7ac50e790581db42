"""Request loop over resident factored systems (tbs_server_* of the C ABI).

``Server`` registers systems once (upload + factorization, kept in HBM) and
takes requests of 1..n right-hand sides, optionally with new Jacobian values
that re-factor the system first.  A thread inside the library admits requests
by device footprint and sweeps every admitted right-hand side together,
letting new requests join at sweep boundaries (continuous batching).  Each
solution is bit-identical to ``Solver.solve`` of the same system and
right-hand side alone.  There is no counterpart in the reference, whose driver
solves one system per run.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .lij import Jacobian, Mesh

STAT_NAMES = ("requests_done", "rhs_done", "graph_launches", "refactors", "peak_rhs_in_flight",
              "peak_rhs_bytes", "resident_system_bytes", "queued", "us_start", "us_members",
              "us_run", "us_retire")


class Request:
    """A submitted request; keeps its arrays alive until ``wait`` returns."""

    def __init__(self, server: "Server", rid: int, nrhs: int, rhs, U, jac_arrays):
        self.server = server
        self.id = rid
        self.nrhs = nrhs
        self._rhs = rhs
        self.U = U
        self._jac = jac_arrays
        self.result = None

    def done(self) -> bool:
        if self.result is not None:
            return True
        d = C.c_int()
        self.server._chk(N.lib.tbs_server_poll(self.server.handle, self.id, C.byref(d)))
        return bool(d.value)

    def wait(self):
        """(U [nrhs, 9 nelem], sweeps [nrhs], rel_residual [nrhs], latency_ms, queue_ms)."""
        if self.result is None:
            sw = np.zeros(self.nrhs, np.int32)
            rel = np.zeros(self.nrhs)
            lat, q = C.c_double(), C.c_double()
            rc = N.lib.tbs_server_wait(self.server.handle, self.id, N.iptr(sw), N.dptr(rel),
                                       C.byref(lat), C.byref(q))
            self._rhs = self._jac = None
            self.server._chk(rc)
            self.result = (self.U, sw, rel, lat.value, q.value)
        return self.result


class Server:
    def __init__(self, device_id: int = 0, algo: int = N.ALGO_FP64, budget_bytes: int = 32 << 30,
                 max_rhs: int = 64, chunk: int | None = None,
                 lane_split: int | list[int] | None = None):
        """lane_split: one cell count (two lanes; 0 = one lane) or an ascending
        list of up to three (default: [262144, 1048576], three lanes)."""
        h = C.c_void_p()
        N.check_server(N.lib.tbs_server_create(device_id, algo, budget_bytes, max_rhs, C.byref(h)))
        self.handle = h
        self.nelem = {}
        try:
            if chunk is not None:
                self.set_chunk(chunk)
            if isinstance(lane_split, (list, tuple)):
                arr = (C.c_longlong * max(len(lane_split), 1))(*lane_split)
                self._chk(N.lib.tbs_server_set_lane_splits(self.handle, arr, len(lane_split)))
            elif lane_split is not None:
                self._chk(N.lib.tbs_server_set_lanes(self.handle, lane_split))
        except Exception:
            self.close()
            raise

    def _chk(self, rc):
        N.check_server(rc, self.handle)

    def set_chunk(self, sweeps: int):
        self._chk(N.lib.tbs_server_set_chunk(self.handle, sweeps))

    def add_system(self, mesh: Mesh, jac: Jacobian) -> int:
        sid = C.c_int()
        f = [np.ascontiguousarray(getattr(mesh, k), np.int32) for k in Mesh.FIELDS]
        self._chk(N.lib.tbs_server_add_system(
            self.handle, mesh.nvar, mesh.nelem, mesh.nintface, mesh.eftot, mesh.nline,
            mesh.nlineelem, *[N.iptr(a) for a in f], N.dptr(jac.jacD), N.dptr(jac.jacO1),
            N.dptr(jac.jacO2), C.byref(sid)))
        self.nelem[sid.value] = mesh.nelem
        return sid.value

    def system_bytes(self, sid: int, max_sweeps: int):
        a, b = C.c_size_t(), C.c_size_t()
        self._chk(N.lib.tbs_server_system_bytes(self.handle, sid, max_sweeps, C.byref(a), C.byref(b)))
        return a.value, b.value

    def submit(self, sid: int, rhs: np.ndarray, rel_tol: float, max_sweeps: int = 200,
               new_jacobian: Jacobian | None = None, out: np.ndarray | None = None) -> Request:
        rhs = np.ascontiguousarray(rhs, np.float64)
        if sid not in self.nelem:
            raise N.TbsError(N.TBS_ERR_ARG, f"unknown system {sid}")
        nv = 9 * self.nelem[sid]
        if rhs.size % nv:
            raise ValueError("rhs must hold whole right-hand sides of 9*nelem entries")
        nrhs = rhs.size // nv
        U = out if out is not None else np.empty((nrhs, nv))
        jac = None
        if new_jacobian is not None:
            jac = (new_jacobian.jacD, new_jacobian.jacO1, new_jacobian.jacO2)
        rid = C.c_longlong()
        self._chk(N.lib.tbs_server_submit(
            self.handle, sid, nrhs, N.dptr(rhs), N.dptr(U), rel_tol, max_sweeps,
            *([N.dptr(a) for a in jac] if jac else [None, None, None]), C.byref(rid)))
        return Request(self, rid.value, nrhs, rhs, U, jac)

    def stats(self) -> dict:
        v = (C.c_longlong * len(STAT_NAMES))()
        self._chk(N.lib.tbs_server_stats(self.handle, v, len(STAT_NAMES)))
        return dict(zip(STAT_NAMES, (int(x) for x in v)))

    def close(self):
        if self.handle:
            N.lib.tbs_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
