"""Python mirror of the reference's host interface for the LIJ path.

``Platform``, ``Mesh`` and ``Jacobian`` keep the member and method names of
the reference's C++ classes (include/Platform.hxx:25-93,
include/Mesh.hxx:27-67, include/Jacobian.hxx:43-98); ``Solver`` is the
device phase of src/main.cxx:180-229 (factor, sweeps, report) over the
C ABI.  Arrays are numpy, 0-based, column-major 9x9 blocks as in the files.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N


class Platform:
    """Device selection (src/Platform.cxx:11-78).  Only compute_mode 2 (CUDA)."""

    def __init__(self, compute_mode: int = N.CUDA_MODE, device_id: int = 0):
        if compute_mode != N.CUDA_MODE:
            raise N.TbsError(N.TBS_ERR_UNSUPPORTED,
                             f"compute_mode {compute_mode} is not available: this build runs "
                             "only on CUDA (mode 2)")
        self.compute_mode = compute_mode
        self.device_id = device_id
        h = C.c_void_p()
        N.check(N.lib.tbs_create(device_id, C.byref(h)))
        self.ctx = h

    def memoryAllocated(self) -> int:
        b = C.c_size_t()
        N.check(N.lib.tbs_memory_allocated(self.ctx, C.byref(b)), self.ctx)
        return b.value

    def close(self):
        if self.ctx:
            N.lib.tbs_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Mesh:
    """Line mesh (include/Mesh.hxx:27-67)."""

    FIELDS = ("epoint", "ef", "fc", "linesize", "linepoint", "lines", "lineface")

    def __init__(self):
        self.nvar = self.nelem = self.nintface = self.eftot = 0
        self.nline = self.nlineelem = self.max_line_nelem = 0
        for f in self.FIELDS:
            setattr(self, f, np.zeros(0, np.int32))
        self._gpu = None

    # ------------------------------------------------------------ construction
    def _alloc(self, hdr):
        (self.nvar, self.nelem, self.nintface, self.eftot,
         self.nline, self.nlineelem) = (int(v) for v in hdr)
        self.epoint = np.zeros(self.nelem + 1, np.int32)
        self.ef = np.zeros(self.eftot, np.int32)
        self.fc = np.zeros(2 * self.nintface, np.int32)
        self.linesize = np.zeros(self.nline, np.int32)
        self.linepoint = np.zeros(self.nline + 1, np.int32)
        self.lines = np.zeros(self.nlineelem, np.int32)
        self.lineface = np.zeros(self.nlineelem, np.int32)

    def _finish(self):
        self.max_line_nelem = int(self.linesize.max()) if self.nline else 0
        self.nbytes = sum(getattr(self, f).size for f in self.FIELDS)

    @property
    def header(self) -> np.ndarray:
        return np.array([self.nvar, self.nelem, self.nintface, self.eftot, self.nline,
                         self.nlineelem], np.int32)

    def _arrays(self):
        return [N.iptr(getattr(self, f)) for f in self.FIELDS]

    def fromFile(self, path: str = "gpuline.mesh.data.bin") -> bool:
        """src/Mesh.cxx:11-73 (raises instead of exit(1))."""
        hdr = np.zeros(6, np.int32)
        N.check(N.lib.tbs_read_mesh_header(path.encode(), N.iptr(hdr)))
        self._alloc(hdr)
        N.check(N.lib.tbs_read_mesh(path.encode(), N.iptr(hdr), *self._arrays()))
        self._finish()
        return True

    @classmethod
    def from_file(cls, path: str = "gpuline.mesh.data.bin") -> "Mesh":
        m = cls()
        m.fromFile(path)
        return m

    @classmethod
    def structured(cls, L: int, K: int, nvar: int = 9) -> "Mesh":
        """L lines of K cells in the numbering of the reference's data sets."""
        m = cls()
        hdr = np.zeros(6, np.int32)
        N.check(N.lib.tbs_gen_structured_header(L, K, nvar, N.iptr(hdr)))
        m._alloc(hdr)
        N.check(N.lib.tbs_gen_structured_mesh(L, K, *m._arrays()))
        m._finish()
        return m

    @classmethod
    def from_arrays(cls, nvar, **arrays) -> "Mesh":
        m = cls()
        for f in cls.FIELDS:
            setattr(m, f, np.ascontiguousarray(arrays[f], np.int32))
        m.nvar = int(nvar)
        m.nelem = m.epoint.size - 1
        m.nintface = m.fc.size // 2
        m.eftot = m.ef.size
        m.nline = m.linesize.size
        m.nlineelem = m.lines.size
        m._finish()
        return m

    def toFile(self, path: str) -> None:
        hdr = self.header
        N.check(N.lib.tbs_write_mesh(path.encode(), N.iptr(hdr), *self._arrays()))

    def validate(self) -> None:
        hdr = self.header
        N.check(N.lib.tbs_validate_mesh(N.iptr(hdr), *self._arrays()))

    # ------------------------------------------------------------------ device
    def setupDevice(self, gpu: Platform) -> None:
        self._gpu = gpu

    def toDevice(self) -> None:
        g = self._gpu
        N.check(N.lib.tbs_set_mesh(g.ctx, self.nvar, self.nelem, self.nintface, self.eftot,
                                   self.nline, self.nlineelem, *self._arrays()), g.ctx)

    def fromDevice(self) -> None:
        """The mesh is never modified on the device."""


class Jacobian:
    """Block Jacobian and vectors (include/Jacobian.hxx:43-98)."""

    def __init__(self):
        self.nvar = self.nelem = self.nintface = 0
        self._gpu = None

    def _alloc(self, nvar, nelem, nintface, nlineelem):
        self.nvar, self.nelem, self.nintface = int(nvar), int(nelem), int(nintface)
        nb = self.nvar * self.nvar
        self.jacD = np.zeros(nb * nelem)
        self.jacDLU = np.zeros(nb * nelem)
        self.jacO1 = np.zeros(nb * nintface)
        self.jacO2 = np.zeros(nb * nintface)
        self.rhs = np.zeros(self.nvar * nelem)
        self.U0 = np.zeros(self.nvar * nelem)
        self.U = np.zeros(self.nvar * nelem)
        self.dU = np.zeros(self.nvar * nelem)
        self.res = np.zeros(self.nvar * nelem)
        self.DinvC = np.zeros(nb * nelem)
        self.A = np.zeros(nb * nlineelem)

    def fromFile(self, nlineelem: int, path: str = "gpuline.jacobian.data.bin") -> bool:
        """src/Jacobian.cxx:11-74."""
        hdr = np.zeros(3, np.int32)
        N.check(N.lib.tbs_read_jacobian_header(path.encode(), N.iptr(hdr)))
        self._alloc(hdr[0], hdr[1], hdr[2], nlineelem)
        N.check(N.lib.tbs_read_jacobian(path.encode(), N.iptr(hdr), N.dptr(self.jacD),
                                        N.dptr(self.jacO1), N.dptr(self.jacO2), N.dptr(self.rhs),
                                        N.dptr(self.U0)))
        return True

    @classmethod
    def generate(cls, mesh: Mesh, shift: float = 9.0, seed: int = 1) -> "Jacobian":
        """Seeded synthetic values: jacD = U(-1,1) + shift I, O = 0.1 U(-1,1), rhs = U(-1,1)."""
        j = cls()
        j._alloc(mesh.nvar, mesh.nelem, mesh.nintface, mesh.nlineelem)
        N.check(N.lib.tbs_gen_jacobian(mesh.nvar, mesh.nelem, mesh.nintface, float(shift),
                                       int(seed), N.dptr(j.jacD), N.dptr(j.jacO1),
                                       N.dptr(j.jacO2), N.dptr(j.rhs), N.dptr(j.U0)))
        return j

    def toFile(self, path: str) -> None:
        hdr = np.array([self.nvar, self.nelem, self.nintface], np.int32)
        N.check(N.lib.tbs_write_jacobian(path.encode(), N.iptr(hdr), N.dptr(self.jacD),
                                         N.dptr(self.jacO1), N.dptr(self.jacO2),
                                         N.dptr(self.rhs), N.dptr(self.U0)))

    def assembleTriBlocks(self, mesh: Mesh) -> None:
        """src/Jacobian.cxx:76-117: A[e] = in-line lower block of row e."""
        nb = self.nvar * self.nvar
        if self.A.size < nb * mesh.nelem:
            self.A = np.zeros(nb * mesh.nelem)
        O1 = self.jacO1.reshape(-1, nb)
        O2 = self.jacO2.reshape(-1, nb)
        A = self.A.reshape(-1, nb)
        for l in range(mesh.nline):
            for k in range(1, int(mesh.linesize[l])):
                m = int(mesh.linepoint[l]) + k
                f = int(mesh.lineface[m])
                e = int(mesh.lines[m])
                A[e] = O2[f] if e == mesh.fc[2 * f] else O1[f]

    def resizeBlockSize(self, nvar_new: int) -> None:
        """src/Jacobian.cxx:153-238 (same resulting arrays)."""
        if nvar_new == self.nvar:
            return
        nb = nvar_new * nvar_new
        D = np.zeros(nb * self.nelem)
        O1 = np.zeros(nb * self.nintface)
        O2 = np.zeros(nb * self.nintface)
        r = np.zeros(nvar_new * self.nelem)
        u0 = np.zeros(nvar_new * self.nelem)
        N.check(N.lib.tbs_resize_block_size(self.nvar, nvar_new, self.nelem, self.nintface,
                                            N.dptr(self.jacD), N.dptr(self.jacO1),
                                            N.dptr(self.jacO2), N.dptr(self.rhs),
                                            N.dptr(self.U0), N.dptr(D), N.dptr(O1), N.dptr(O2),
                                            N.dptr(r), N.dptr(u0)))
        self.nvar = nvar_new
        self.jacD, self.jacO1, self.jacO2, self.rhs, self.U0 = D, O1, O2, r, u0
        self.U = np.zeros(nvar_new * self.nelem)
        self.dU = np.zeros(nvar_new * self.nelem)
        self.res = np.zeros(nvar_new * self.nelem)
        self.jacDLU = np.zeros(nb * self.nelem)
        self.A = np.zeros(nb * self.nelem)

    def setupDevice(self, gpu: Platform) -> None:
        self._gpu = gpu

    def toDevice(self) -> None:
        g = self._gpu
        N.check(N.lib.tbs_set_jacobian(g.ctx, N.dptr(self.jacD), N.dptr(self.jacO1),
                                       N.dptr(self.jacO2), N.dptr(self.rhs), N.dptr(self.U0)),
                g.ctx)

    def fromDevice(self) -> None:
        g = self._gpu
        N.check(N.lib.tbs_get_solution(g.ctx, N.dptr(self.U)), g.ctx)
        N.check(N.lib.tbs_get_residual(g.ctx, N.dptr(self.res)), g.ctx)
        N.check(N.lib.tbs_get_update(g.ctx, N.dptr(self.dU)), g.ctx)


class Solver:
    """One device context: upload, factor, sweep, solve, read back."""

    def __init__(self, device_id: int = 0, platform: Platform | None = None):
        self.platform = platform or Platform(N.CUDA_MODE, device_id)
        self.ctx = self.platform.ctx
        self.nvar = self.nelem = 0
        self._staged = []  # host arrays of staged systems, oldest first

    def _chk(self, rc):
        N.check(rc, self.ctx)

    def set_stream(self, stream_handle: int | None):
        self._chk(N.lib.tbs_set_stream(self.ctx, stream_handle))

    def set_mesh(self, mesh: Mesh):
        mesh.setupDevice(self.platform)
        mesh.toDevice()
        self.nvar, self.nelem = mesh.nvar, mesh.nelem
        self._staged = []

    def set_jacobian(self, jac: Jacobian):
        jac.setupDevice(self.platform)
        jac.toDevice()
        self._staged = []

    def set_jacobian_arrays(self, jacD, jacO1, jacO2, rhs):
        self._chk(N.lib.tbs_set_jacobian(self.ctx, N.dptr(jacD), N.dptr(jacO1), N.dptr(jacO2),
                                         N.dptr(rhs), None))
        self._staged = []  # discarded by the call

    def stage_jacobian_arrays(self, jacD, jacO1, jacO2, rhs):
        """Upload a coming system's Jacobian and rhs while the current one is
        solved; up to two may wait, and each ``factor`` switches to the older
        one.  Pass pinned host arrays for the copy to overlap, and keep them
        unchanged until that ``factor`` returns (this object holds
        references until then)."""
        arrs = [np.ascontiguousarray(a, np.float64) for a in (jacD, jacO1, jacO2, rhs)]
        self._chk(N.lib.tbs_stage_jacobian(self.ctx, *[N.dptr(a) for a in arrs]))
        self._staged.append(arrs)

    def set_jacobian_device(self, d_jacD: int, d_jacO1: int, d_jacO2: int, d_rhs: int):
        self._chk(N.lib.tbs_set_jacobian_device(self.ctx, d_jacD, d_jacO1, d_jacO2, d_rhs))
        self._staged = []

    def set_rhs(self, rhs: np.ndarray):
        self._chk(N.lib.tbs_set_rhs(self.ctx, N.dptr(np.ascontiguousarray(rhs, np.float64))))

    def set_initial(self, U: np.ndarray | None):
        self._chk(N.lib.tbs_set_initial(
            self.ctx, None if U is None else N.dptr(np.ascontiguousarray(U, np.float64))))

    def set_inner_sweeps(self, m: int):
        self._chk(N.lib.tbs_set_inner_sweeps(self.ctx, m))

    def set_inner_schedule(self, first: int, rest: int):
        """TBS_ALGO_MIXED: `first` inner sweeps in a solve's first outer step, `rest` after."""
        self._chk(N.lib.tbs_set_inner_schedule(self.ctx, first, rest))

    def inner_schedule(self):
        f, r = C.c_int(), C.c_int()
        self._chk(N.lib.tbs_get_inner_schedule(self.ctx, C.byref(f), C.byref(r)))
        return f.value, r.value

    def tune_inner(self, rel_tol: float, max_sweeps: int = 100):
        """Pick the fastest FP32 inner sweep schedule for TBS_ALGO_MIXED (device timing);
        returns (steady inner sweeps, ms); inner_schedule() gives the first step's too."""
        m = C.c_int()
        ms = C.c_double()
        self._chk(N.lib.tbs_tune_inner(self.ctx, rel_tol, max_sweeps, C.byref(m), C.byref(ms)))
        return m.value, ms.value

    def factor(self, algo: int = N.ALGO_FP64):
        self._chk(N.lib.tbs_factor(self.ctx, algo))
        if self._staged:
            self._staged.pop(0)

    def sweep(self, n: int) -> np.ndarray:
        h = np.zeros(n + 1)
        self._chk(N.lib.tbs_sweep(self.ctx, n, N.dptr(h)))
        return h

    def solve(self, rel_tol: float, max_sweeps: int = 1000):
        h = np.zeros(max_sweeps + 1)
        s = C.c_int()
        self._chk(N.lib.tbs_solve(self.ctx, rel_tol, max_sweeps, C.byref(s), N.dptr(h)))
        return s.value, h[: s.value + 1]

    def gmres(self, rel_tol: float, restart: int = 30, precond_sweeps: int = 1,
              max_iters: int = 300):
        """Line-preconditioned restarted GMRES on J U = -rhs (ALGO_FP64 factors).
        Returns (Arnoldi steps, residual history); the solution is in ``solution()``."""
        h = np.zeros(max_iters + 1)
        it = C.c_int()
        self._chk(N.lib.tbs_gmres(self.ctx, restart, precond_sweeps, rel_tol, max_iters,
                                  C.byref(it), N.dptr(h)))
        return it.value, h[: it.value + 1]

    def solve_multi(self, rhs: np.ndarray, rel_tol: float, max_sweeps: int = 1000, out=None):
        """Several right-hand sides (rows of ``rhs``, 9*nelem each) from U = 0
        with the current factors (ALGO_FP64), groups of up to 8 sweeping
        together.  Returns (U [nrhs, 9*nelem], sweeps [nrhs], list of norm
        histories); each row equals ``set_rhs`` + ``solve`` of it alone.
        ``out``: a C-contiguous float64 [nrhs, 9*nelem] array to receive U
        (pinned host memory makes the device-to-host copy direct)."""
        n = self.nvar * self.nelem
        rhs = np.ascontiguousarray(rhs, np.float64).reshape(-1, n)
        nrhs = rhs.shape[0]
        if out is None:
            U = np.zeros((nrhs, n))
        elif out.dtype != np.float64 or out.size != nrhs * n or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous float64 array of {nrhs} x {n} values")
        else:
            U = out.reshape(nrhs, n)
        sw = np.zeros(nrhs, np.int32)
        h = np.zeros((nrhs, max_sweeps + 1))
        self._chk(N.lib.tbs_solve_multi(self.ctx, nrhs, N.dptr(rhs), N.dptr(U), rel_tol,
                                        max_sweeps, N.iptr(sw), N.dptr(h), max_sweeps + 1))
        return U, sw, [h[r, : sw[r] + 1].copy() for r in range(nrhs)]

    def solve_multi_device(self, d_rhs: int, d_U: int, nrhs: int, rel_tol: float,
                           max_sweeps: int = 1000):
        """``solve_multi`` on device buffers (addresses of nrhs * 9*nelem
        doubles, element order).  Returns (sweeps [nrhs], norm histories)."""
        sw = np.zeros(nrhs, np.int32)
        h = np.zeros((nrhs, max_sweeps + 1))
        self._chk(N.lib.tbs_solve_multi_device(self.ctx, nrhs, d_rhs, d_U, rel_tol, max_sweeps,
                                               N.iptr(sw), N.dptr(h), max_sweeps + 1))
        return sw, [h[r, : sw[r] + 1].copy() for r in range(nrhs)]

    def _vec(self, fn, out=None):
        """``out``: a C-contiguous float64 array of nvar*nelem to fill (pinned
        host memory makes the device-to-host copy direct); default a new one."""
        n = self.nvar * self.nelem
        if out is None:
            out = np.zeros(n)
        elif out.dtype != np.float64 or out.size != n or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous float64 array of {n} values")
        self._chk(fn(self.ctx, N.dptr(out)))
        return out

    def solution(self, out=None) -> np.ndarray:
        return self._vec(N.lib.tbs_get_solution, out)

    def residual(self, out=None) -> np.ndarray:
        return self._vec(N.lib.tbs_get_residual, out)

    def update(self, out=None) -> np.ndarray:
        return self._vec(N.lib.tbs_get_update, out)

    def true_residual_norm(self) -> float:
        v = C.c_double()
        self._chk(N.lib.tbs_true_residual_norm(self.ctx, C.byref(v)))
        return v.value

    def resid_timer(self, reset: bool = False):
        """(total microseconds, launches) of the sweeps' residual launches on
        the device clock since the last reset; reset=True starts anew."""
        us, n = C.c_double(), C.c_longlong()
        self._chk(N.lib.tbs_resid_timer(self.ctx, C.byref(us), C.byref(n), 1 if reset else 0))
        return us.value, n.value

    def set_check(self, on: bool = True):
        """TBS_ALGO_FP64: check a converged solve against rhs + J U (default on)."""
        self._chk(N.lib.tbs_set_check(self.ctx, 1 if on else 0))

    def solve_check(self):
        """(true residual norm at the last check or -1, checks, restarts) of the last solve."""
        t, c, r = C.c_double(), C.c_int(), C.c_int()
        self._chk(N.lib.tbs_solve_check(self.ctx, C.byref(t), C.byref(c), C.byref(r)))
        return t.value, c.value, r.value

    def update_values(self, jacD, jacO1, jacO2):
        """New block values for the residual, the factorization kept (a lagged
        factorization): the solve converges to the new system."""
        a = [np.ascontiguousarray(x, np.float64) for x in (jacD, jacO1, jacO2)]
        self._chk(N.lib.tbs_update_values(self.ctx, *[N.dptr(x) for x in a]))

    def profile(self, on: bool = True):
        self._chk(N.lib.tbs_profile_enable(self.ctx, 1 if on else 0))

    def profile_reset(self):
        self._chk(N.lib.tbs_profile_reset(self.ctx))

    def profile_read(self) -> dict:
        n = C.c_int(16)
        names = (C.c_char_p * 16)()
        launches = (C.c_longlong * 16)()
        ms = (C.c_double * 16)()
        self._chk(N.lib.tbs_profile_read(self.ctx, C.byref(n), names, launches, ms))
        return {names[i].decode(): (int(launches[i]), float(ms[i])) for i in range(n.value)}

    def kernel_bytes(self, name: str) -> float:
        v = C.c_double()
        self._chk(N.lib.tbs_kernel_bytes(self.ctx, name.encode(), C.byref(v)))
        return v.value

    def memory_allocated(self) -> int:
        return self.platform.memoryAllocated()

    def close(self):
        self.platform.close()


class Batch:
    """Independent systems (factored Solvers on one GPU) solved together.

    ``solve`` runs one CUDA graph launch in which every sweep is a persistent
    Thomas launch over the lines of all unconverged systems (device work
    queue, longest lines first), a residual launch over their tiles and a
    per-system norm launch.  Each system stops at its own tolerance, and its
    iterates are bit-identical to ``Solver.solve`` on it alone.
    """

    def __init__(self, solvers: list[Solver]):
        if not solvers:
            raise ValueError("a batch needs at least one system")
        self.solvers = list(solvers)
        arr = (C.c_void_p * len(solvers))(*[s.ctx for s in solvers])
        h = C.c_void_p()
        N.check_batch(N.lib.tbs_batch_create(arr, len(solvers), C.byref(h)))
        self.handle = h

    def _chk(self, rc):
        N.check_batch(rc, self.handle)

    def __len__(self):
        return len(self.solvers)

    def solve(self, rel_tol: float, max_sweeps: int = 1000):
        """Returns (sweeps per system, list of per-system norm histories)."""
        n = len(self.solvers)
        sw = np.zeros(n, np.int32)
        h = np.zeros((n, max_sweeps + 1))
        self._chk(N.lib.tbs_batch_solve(self.handle, rel_tol, max_sweeps, N.iptr(sw), N.dptr(h)))
        return sw, [h[s, : sw[s] + 1].copy() for s in range(n)]

    def set_stream(self, stream_handle: int | None):
        self._chk(N.lib.tbs_batch_set_stream(self.handle, stream_handle))

    def set_schedule(self, ctas_per_sm: int, stages: int, order: int = 0):
        self._chk(N.lib.tbs_batch_set_schedule(self.handle, ctas_per_sm, stages, order))

    def schedule(self):
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        self._chk(N.lib.tbs_batch_get_schedule(self.handle, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def set_warps_per_line(self, warps: int):
        """1: the chain warp issues its own staging copies; 2: a copy warp per line."""
        self._chk(N.lib.tbs_batch_set_warps_per_line(self.handle, warps))

    def warps_per_line(self) -> int:
        w = C.c_int()
        self._chk(N.lib.tbs_batch_get_warps_per_line(self.handle, C.byref(w)))
        return w.value

    def tune(self):
        """Autotune the persistent Thomas launch (warps per line, CTAs per SM,
        stages, line order); returns (ctas_per_sm, stages, order, ms);
        warps_per_line() gives the tuned warps."""
        a, b, c, ms = C.c_int(), C.c_int(), C.c_int(), C.c_double()
        self._chk(N.lib.tbs_batch_tune(self.handle, C.byref(a), C.byref(b), C.byref(c),
                                       C.byref(ms)))
        return a.value, b.value, c.value, ms.value

    def set_inner_sweeps(self, m: int):
        self._chk(N.lib.tbs_batch_set_inner_sweeps(self.handle, m))

    def tune_inner(self, rel_tol: float, max_sweeps: int = 200):
        """ALGO_MIXED: pick the fastest inner sweep schedule with which every
        member reaches rel_tol (device timing); returns (first, rest, ms)."""
        f, r, ms = C.c_int(), C.c_int(), C.c_double()
        self._chk(N.lib.tbs_batch_tune_inner(self.handle, rel_tol, max_sweeps, C.byref(f),
                                             C.byref(r), C.byref(ms)))
        return f.value, r.value, ms.value

    def set_inner_schedule(self, first: int, rest: int):
        self._chk(N.lib.tbs_batch_set_inner_schedule(self.handle, first, rest))

    def profile(self, on: bool = True):
        self._chk(N.lib.tbs_batch_profile_enable(self.handle, 1 if on else 0))

    def profile_reset(self):
        self._chk(N.lib.tbs_batch_profile_reset(self.handle))

    def profile_read(self) -> dict:
        n = C.c_int(16)
        names = (C.c_char_p * 16)()
        launches = (C.c_longlong * 16)()
        ms = (C.c_double * 16)()
        self._chk(N.lib.tbs_batch_profile_read(self.handle, C.byref(n), names, launches, ms))
        return {names[i].decode(): (int(launches[i]), float(ms[i])) for i in range(n.value)}

    def close(self):
        if self.handle:
            N.lib.tbs_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
