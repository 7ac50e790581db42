"""CPU oracle of the reference LIJ path -- TEST INFRASTRUCTURE ONLY.

ctypes wrapper of ``oracle/_build/liboracle.so`` (built from lij_oracle.c by
oracle/Makefile).  Only the tests, ``__graft_entry__.smoke()`` and the CPU
baseline / reference arm of ``bench.py`` use it, and only as the checker or
as the timed CPU baseline; the product (libtriblock.so) never does.

Parity status: the arithmetic restatement is unpinned by reference outputs
(the reference needs OCCA, MPI and gfortran to build and ships no golden
vectors); the mesh format is pinned by the ex05 fixture in tests/golden.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")


def _load():
    if not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", HERE], check=True, capture_output=True)
    return C.CDLL(LIB_PATH)


lib = _load()
_i, _ip, _dp = C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)
lib.oracle_set_threads.argtypes = [_i]
lib.oracle_max_threads.restype = _i
lib.oracle_lij.restype = _i
lib.oracle_lij.argtypes = [_i, _i, _i, _i] + [_ip] * 7 + [_dp] * 4 + [_i] + [_dp] * 6
lib.oracle_norm.restype = C.c_double
lib.oracle_norm.argtypes = [_dp, C.c_size_t]
lib.oracle_resize_block_size.argtypes = [_i, _i, _i, _i] + [_dp] * 10
lib.oracle_line_res.argtypes = [_i, _i] + [_ip] * 6 + [_dp] * 5
lib.oracle_solve_du.argtypes = [_i, _i] + [_ip] * 3 + [_dp] * 5
lib.oracle_line_lu.argtypes = [_i, _i] + [_ip] * 5 + [_dp] * 4
lib.oracle_assemble_A.argtypes = [_i, _i] + [_ip] * 5 + [_dp] * 3
lib.oracle_factor.restype = _i
lib.oracle_factor.argtypes = [_i, _i, _i] + [_ip] * 5 + [_dp] * 6
lib.oracle_sweeps.restype = _i
lib.oracle_sweeps.argtypes = [_i, _i, _i] + [_ip] * 6 + [_dp] * 10 + [_i, _dp]


def _ip_(a):
    a = np.ascontiguousarray(a, np.int32)
    return a, a.ctypes.data_as(_ip)


def _dp_(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def set_threads(n: int) -> None:
    lib.oracle_set_threads(int(n))


def max_threads() -> int:
    return int(lib.oracle_max_threads())


def lij(mesh, jacD, jacO1, jacO2, rhs, iters: int, threads: int = 1, want_factors=False):
    """The reference flow (src/main.cxx:180-229) for `iters` sweeps from U = 0.

    `mesh` has the reference's 0-based arrays (epoint, ef, fc, linesize,
    linepoint, lines, lineface) and nvar / nelem / nintface / nline.
    Returns dict(U, R, dU, hist[, DLU, DinvC]).
    """
    set_threads(threads)
    nv, ne = int(mesh.nvar), int(mesh.nelem)
    keep = []
    ptrs = []
    for f in ("epoint", "ef", "fc", "linesize", "linepoint", "lines", "lineface"):
        a, p = _ip_(getattr(mesh, f))
        keep.append(a)
        ptrs.append(p)
    U = np.zeros(nv * ne)
    R = np.zeros(nv * ne)
    dU = np.zeros(nv * ne)
    hist = np.zeros(iters + 1)
    DLU = np.zeros(nv * nv * ne) if want_factors else None
    DinvC = np.zeros(nv * nv * ne) if want_factors else None
    rc = lib.oracle_lij(nv, ne, int(mesh.nintface), int(mesh.nline), *ptrs,
                        _dp_(jacD), _dp_(jacO1), _dp_(jacO2), _dp_(rhs), int(iters),
                        _dp_(U), _dp_(R), _dp_(dU), _dp_(hist),
                        _dp_(DLU) if want_factors else None,
                        _dp_(DinvC) if want_factors else None)
    if rc != 0:
        raise RuntimeError(f"oracle_lij failed ({rc})")
    out = dict(U=U, R=R, dU=dU, hist=hist)
    if want_factors:
        out.update(DLU=DLU, DinvC=DinvC)
    return out


# ---------------------------------------------------------------------------
# oracle/_ref: the reference's own kernels (OKL translated by okl2c.py) driven
# in src/main.cxx order.  Built here by `make -C oracle ref REFERENCE=<checkout>`
# (needs the reference checkout); the built library travels with the tree.
REF_LIB_PATH = os.path.join(HERE, "_ref", "libokl_ref.so")
_ref_lib = None


def ref_available() -> bool:
    return os.path.exists(REF_LIB_PATH)


def build_ref(reference_dir: str) -> str:
    """Translates and compiles the reference's kernels into oracle/_ref."""
    subprocess.run(["make", "-C", HERE, "ref", f"REFERENCE={reference_dir}"], check=True,
                   capture_output=True)
    return REF_LIB_PATH


def _ref():
    global _ref_lib
    if _ref_lib is None:
        if not ref_available():
            raise FileNotFoundError(f"{REF_LIB_PATH} is not built (make -C oracle ref "
                                    "REFERENCE=<reference checkout>)")
        L = C.CDLL(REF_LIB_PATH)
        L.okl_ref_set_threads.argtypes = [_i]
        L.okl_ref_lij.restype = _i
        L.okl_ref_lij.argtypes = [_i] * 7 + [_ip] * 7 + [_dp] * 4 + [_i] + [_dp] * 10
        L.okl_ref_true_residual.restype = _i
        L.okl_ref_true_residual.argtypes = [_i] * 7 + [_ip] * 6 + [_dp] * 6
        L.okl_ref_factor.restype = C.c_void_p
        L.okl_ref_factor.argtypes = [_i] * 7 + [_ip] * 7 + [_dp] * 4
        L.okl_ref_sweeps.argtypes = [C.c_void_p, _dp, _dp, _dp, _i]
        L.okl_ref_free.argtypes = [C.c_void_p]
        L.okl_ref_assemble_tri_blocks.argtypes = [_i] * 5 + [_ip] * 5 + [_dp] * 3
        L.okl_ref_resize_block_size.argtypes = [_i] * 4 + [_dp] * 10
        _ref_lib = L
    return _ref_lib


def _mesh_sizes(mesh):
    linesize = np.asarray(mesh.linesize)
    nlineelem = int(getattr(mesh, "nlineelem", int(linesize.sum())))
    mx = int(getattr(mesh, "max_line_nelem", int(linesize.max()) if linesize.size else 1))
    return (int(mesh.nvar), int(mesh.nelem), int(mesh.nintface), int(mesh.eftot),
            int(mesh.nline), max(nlineelem, int(mesh.nelem)), max(mx, 1))


def ref_lij(mesh, jacD, jacO1, jacO2, rhs, iters: int, threads: int = 1, per_sweep=False,
            want_factors=False):
    """The reference's own kernels for `iters` sweeps from U = 0.
    Returns dict(U, R, dU, hist[, U_all, R_all, dU_all][, DLU, DinvC, A])."""
    L = _ref()
    L.okl_ref_set_threads(int(threads))
    sz = _mesh_sizes(mesh)
    nv, ne = sz[0], sz[1]
    keep, ptrs = [], []
    for f in ("epoint", "ef", "fc", "linesize", "linepoint", "lines", "lineface"):
        a, p = _ip_(getattr(mesh, f))
        keep.append(a)
        ptrs.append(p)
    n = nv * ne
    U, R, dU, hist = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(iters + 1)
    alls = [np.zeros((iters, n)) for _ in range(3)] if per_sweep else [None] * 3
    fac = [np.zeros(nv * nv * ne), np.zeros(nv * nv * ne), np.zeros(nv * nv * sz[5])] \
        if want_factors else [None] * 3
    rc = L.okl_ref_lij(*sz, *ptrs, _dp_(np.ascontiguousarray(jacD)), _dp_(np.ascontiguousarray(jacO1)),
                       _dp_(np.ascontiguousarray(jacO2)), _dp_(np.ascontiguousarray(rhs)),
                       int(iters), _dp_(U), _dp_(R), _dp_(dU), _dp_(hist),
                       *[_dp_(a) if a is not None else None for a in fac],
                       *[_dp_(a) if a is not None else None for a in alls])
    if rc != 0:
        raise RuntimeError(f"okl_ref_lij failed ({rc})")
    out = dict(U=U, R=R, dU=dU, hist=hist)
    if per_sweep:
        out.update(U_all=alls[0], R_all=alls[1], dU_all=alls[2])
    if want_factors:
        out.update(DLU=fac[0], DinvC=fac[1], A=fac[2])
    return out


def ref_true_residual(mesh, jacD, jacO1, jacO2, rhs, U):
    """rhs + J U by the reference's own triblock_lineRes."""
    L = _ref()
    sz = _mesh_sizes(mesh)
    keep, ptrs = [], []
    for f in ("epoint", "ef", "fc", "linesize", "linepoint", "lines"):
        a, p = _ip_(getattr(mesh, f))
        keep.append(a)
        ptrs.append(p)
    R = np.zeros(sz[0] * sz[1])
    rc = L.okl_ref_true_residual(*sz, *ptrs, _dp_(np.ascontiguousarray(jacD)),
                                 _dp_(np.ascontiguousarray(jacO1)), _dp_(np.ascontiguousarray(jacO2)),
                                 _dp_(np.ascontiguousarray(rhs, np.float64)),
                                 _dp_(np.ascontiguousarray(U, np.float64)), _dp_(R))
    if rc != 0:
        raise RuntimeError(f"okl_ref_true_residual failed ({rc})")
    return R


def ref_resize_block_size(nv_old, nv_new, nelem, nintface, D, O1, O2, rhs, U0):
    """The reference's own Jacobian::resizeBlockSize; returns (D, O1, O2, rhs, U0)."""
    L = _ref()
    bn = nv_new * nv_new
    out = [np.zeros(bn * nelem), np.zeros(bn * nintface), np.zeros(bn * nintface),
           np.zeros(nv_new * nelem), np.zeros(nv_new * nelem)]
    L.okl_ref_resize_block_size(nv_old, nv_new, nelem, nintface, _dp_(D), _dp_(O1), _dp_(O2),
                                _dp_(rhs), _dp_(U0), *[_dp_(a) for a in out])
    return out


class RefBaseline:
    """The reference's own kernels, factored once, swept on demand: the
    `kind: reference` CPU baseline (OpenMP over lines, OCCA's OpenMP mode)."""

    def __init__(self, mesh, jacD, jacO1, jacO2, rhs, threads: int):
        self.L = _ref()
        self.L.okl_ref_set_threads(int(threads))
        sz = _mesh_sizes(mesh)
        self.n = sz[0] * sz[1]
        self._ints = {f: np.ascontiguousarray(getattr(mesh, f), np.int32) for f in
                      ("epoint", "ef", "fc", "linesize", "linepoint", "lines", "lineface")}
        self._arrs = [np.ascontiguousarray(a, np.float64) for a in (jacD, jacO1, jacO2, rhs)]
        ip = [self._ints[f].ctypes.data_as(_ip) for f in
              ("epoint", "ef", "fc", "linesize", "linepoint", "lines", "lineface")]
        self.h = self.L.okl_ref_factor(*sz, *ip, *[_dp_(a) for a in self._arrs])
        if not self.h:
            raise RuntimeError("okl_ref_factor failed")
        self.reset()

    def reset(self):
        self.U, self.dU = np.zeros(self.n), np.zeros(self.n)
        self.R = self._arrs[3].copy()

    def sweeps(self, n: int) -> None:
        self.L.okl_ref_sweeps(self.h, _dp_(self.U), _dp_(self.R), _dp_(self.dU), int(n))

    def close(self):
        if self.h:
            self.L.okl_ref_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def point_lines(mesh):
    """The mesh with every cell as its own line, faces unchanged.

    The reference's line sweep (src/main.cxx:180-229) on it solves the
    diagonal block alone per cell, dU = -D^-1 R (LU of lineLU_v2.okl:17-27,
    solveLU of :30-52), then U += dU and R = rhs + J U over all faces: the
    point-implicit Jacobi sweep of the paper (p.10-11, Table 4), which the
    reference repository has no code for.  lineface is never read for the
    first cell of a line, so it holds boundary markers."""
    from types import SimpleNamespace
    n = int(mesh.nelem)
    return SimpleNamespace(
        nvar=int(mesh.nvar), nelem=n, nintface=int(mesh.nintface), eftot=int(mesh.eftot),
        nline=n, nlineelem=n, max_line_nelem=1 if n else 0,
        epoint=np.ascontiguousarray(mesh.epoint, np.int32),
        ef=np.ascontiguousarray(mesh.ef, np.int32), fc=np.ascontiguousarray(mesh.fc, np.int32),
        linesize=np.ones(n, np.int32), linepoint=np.arange(n + 1, dtype=np.int32),
        lines=np.arange(n, dtype=np.int32), lineface=np.full(n, -1, np.int32))


def pij(mesh, jacD, jacO1, jacO2, rhs, iters: int, threads: int = 1):
    """Point-implicit Jacobi for `iters` sweeps from U = 0 in the reference's
    operation order: the line sweep on point_lines(mesh).  Returns
    dict(U, R, dU, hist) like lij."""
    return lij(point_lines(mesh), jacD, jacO1, jacO2, rhs, iters, threads)


def gmres(mesh, jacD, jacO1, jacO2, rhs, restart: int, precond_sweeps: int, tol: float,
          max_iters: int, threads: int = 1):
    """Restarted GMRES(restart) on J U = -rhs from U = 0, right preconditioned
    by `precond_sweeps` line sweeps from zero (the paper's line-preconditioned
    GMRES, p.14 Table 6; no code for it in the reference repository).

    The preconditioner is the reference's own sweep loop (lij with rhs = v,
    U after k sweeps ~ -J^-1 v) and the product with J its residual rule
    (true_residual with rhs = 0).  Arnoldi with classical Gram-Schmidt done
    twice, the preconditioned directions kept, Givens rotations for the
    least-squares problem, the true residual recomputed at every restart.
    Returns dict(U, iters, hist) with hist as tbs_gmres fills it."""
    n = rhs.size
    zero = np.zeros(n)

    def P(v):
        return lij(mesh, jacD, jacO1, jacO2, v, precond_sweeps, threads)["U"]

    def J(z, b=zero):
        return true_residual(mesh, jacD, jacO1, jacO2, b, z)

    U = np.zeros(n)
    R = np.array(rhs, dtype=np.float64)
    beta0 = float(np.linalg.norm(R))
    hist = [beta0]
    beta, iters = beta0, 0
    m = restart
    while beta > tol * beta0 and np.isfinite(beta) and iters < max_iters:
        V = [-R / beta]
        Z = []
        H = np.zeros((m + 1, m))
        cs, sn = np.zeros(m), np.zeros(m)
        g = np.zeros(m + 1)
        g[0] = beta
        j = 0
        stop = False
        while j < m and not stop:
            Z.append(P(V[j]))
            w = J(Z[j])
            Vm = np.array(V)
            h1 = Vm @ w
            w = w - Vm.T @ h1
            h2 = Vm @ w
            ww = float(w @ w)
            w = w - Vm.T @ h2
            H[: j + 1, j] = h1 + h2
            hn = np.sqrt(max(ww - float(h2 @ h2), 0.0))
            H[j + 1, j] = hn
            for i in range(j):
                a, b = H[i, j], H[i + 1, j]
                H[i, j], H[i + 1, j] = cs[i] * a + sn[i] * b, -sn[i] * a + cs[i] * b
            a, b = H[j, j], H[j + 1, j]
            r = np.hypot(a, b)
            cs[j], sn[j] = (a / r, b / r) if r > 0 else (1.0, 0.0)
            H[j, j], H[j + 1, j] = r, 0.0
            g[j + 1] = -sn[j] * g[j]
            g[j] = cs[j] * g[j]
            iters += 1
            res = abs(g[j + 1])
            hist.append(res)
            j += 1
            if res <= tol * beta0 or iters >= max_iters or not hn > 0 or not np.isfinite(res):
                stop = True
            elif j < m:
                V.append(w / hn)
        y = np.zeros(j)
        for i in range(j - 1, -1, -1):
            y[i] = (g[i] - H[i, i + 1:j] @ y[i + 1:j]) / H[i, i] if H[i, i] != 0 else 0.0
        U = U + np.array(Z[:j]).T @ y
        R = J(U, rhs)
        beta = float(np.linalg.norm(R))
        hist[iters] = beta
    return dict(U=U, iters=iters, hist=np.array(hist))


def resize_block_size(nv_old, nv_new, nelem, nintface, D, O1, O2, rhs, U0):
    """Jacobian.cxx:153-238 restated; returns the new (D, O1, O2, rhs, U0)."""
    bn = nv_new * nv_new
    out = [np.zeros(bn * nelem), np.zeros(bn * nintface), np.zeros(bn * nintface),
           np.zeros(nv_new * nelem), np.zeros(nv_new * nelem)]
    lib.oracle_resize_block_size(nv_old, nv_new, nelem, nintface, _dp_(D), _dp_(O1), _dp_(O2),
                                 _dp_(rhs), _dp_(U0), *[_dp_(a) for a in out])
    return out


def true_residual(mesh, jacD, jacO1, jacO2, rhs, U):
    """rhs + J U with the reference's residual rule (linesmoothLU_TriBlock_v3.okl:228-336)."""
    nv, ne = int(mesh.nvar), int(mesh.nelem)
    R = np.ascontiguousarray(rhs, np.float64).copy()
    keep, ptrs = [], []
    for f in ("epoint", "ef", "fc", "linesize", "linepoint", "lines"):
        a, p = _ip_(getattr(mesh, f))
        keep.append(a)
        ptrs.append(p)
    U = np.ascontiguousarray(U, np.float64)
    lib.oracle_line_res(nv, int(mesh.nline), *ptrs, _dp_(jacD), _dp_(jacO1), _dp_(jacO2),
                        _dp_(U), _dp_(R))
    return R


class Baseline:
    """Factor once, then time sweeps: the CPU baseline of bench.py.

    Runs the restated reference path (oracle_factor + oracle_sweeps) with
    `threads` OpenMP threads over lines, the work split of the reference's
    OpenMP mode (compute_mode 4)."""

    def __init__(self, mesh, jacD, jacO1, jacO2, rhs, threads: int):
        set_threads(threads)
        self.nv, self.ne, self.nline = int(mesh.nvar), int(mesh.nelem), int(mesh.nline)
        self._ints = {f: np.ascontiguousarray(getattr(mesh, f), np.int32) for f in
                      ("epoint", "ef", "fc", "linesize", "linepoint", "lines", "lineface")}
        self.jacD, self.jacO1, self.jacO2, self.rhs = jacD, jacO1, jacO2, rhs
        nb = self.nv * self.nv * self.ne
        self.DLU, self.DinvC, self.A = np.zeros(nb), np.zeros(nb), np.zeros(nb)
        ip = lambda f: self._ints[f].ctypes.data_as(_ip)
        lib.oracle_factor(self.nv, self.ne, self.nline, ip("fc"), ip("linesize"), ip("linepoint"),
                          ip("lines"), ip("lineface"), _dp_(jacD), _dp_(jacO1), _dp_(jacO2),
                          _dp_(self.DLU), _dp_(self.DinvC), _dp_(self.A))
        self.reset()

    def reset(self):
        self.U = np.zeros(self.nv * self.ne)
        self.dU = np.zeros(self.nv * self.ne)
        self.R = np.array(self.rhs, np.float64, copy=True)

    def sweeps(self, n: int) -> np.ndarray:
        ip = lambda f: self._ints[f].ctypes.data_as(_ip)
        hist = np.zeros(max(n, 1))
        lib.oracle_sweeps(self.nv, self.ne, self.nline, ip("epoint"), ip("ef"), ip("fc"),
                          ip("linesize"), ip("linepoint"), ip("lines"), _dp_(self.jacD),
                          _dp_(self.jacO1), _dp_(self.jacO2), _dp_(self.rhs), _dp_(self.DLU),
                          _dp_(self.DinvC), _dp_(self.A), _dp_(self.U), _dp_(self.R),
                          _dp_(self.dU), int(n), _dp_(hist))
        return hist[:n]
