"""ctypes binding of libtriblock.so (the C ABI declared in include/triblock.h).

The shared library is built in-tree (``triblocksolve_b200/lib``) by
``triblocksolve_b200.build.build_all()``.  There is no CPU implementation of
the solver: if the library is missing, importing this module raises, and every
solver call needs a CUDA device.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
REPO_DIR = os.path.dirname(PKG_DIR)
LIB_PATH = os.path.join(PKG_DIR, "lib", "libtriblock.so")
HEADER_PATH = os.path.join(REPO_DIR, "include", "triblock.h")

TBS_OK = 0
TBS_ERR_ARG = 1
TBS_ERR_IO = 2
TBS_ERR_FORMAT = 3
TBS_ERR_CUDA = 4
TBS_ERR_STATE = 5
TBS_ERR_NUMERIC = 6
TBS_ERR_UNSUPPORTED = 7
TBS_ERR_NOMEM = 8

ALGO_REFERENCE = 0
ALGO_FP64 = 1
ALGO_MIXED = 2
ALGO_PIJ = 3

CUDA_MODE = 2

VEC_SOLUTION = 0  # TBS_VEC_SOLUTION
VEC_UPDATE = 2    # TBS_VEC_UPDATE

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `make -C triblocksolve_b200/csrc` "
        "(or __graft_entry__.build()); there is no CPU fallback")

lib = C.CDLL(LIB_PATH)

_i = C.c_int
_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)
_vp = C.c_void_p
_cp = C.c_char_p


def _sig(name, res, *args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


_sig("tbs_last_error", _cp, _vp)
_sig("tbs_version", _cp)
_sig("tbs_read_mesh_header", _i, _cp, _ip)
_sig("tbs_read_mesh", _i, _cp, _ip, _ip, _ip, _ip, _ip, _ip, _ip, _ip)
_sig("tbs_write_mesh", _i, _cp, _ip, _ip, _ip, _ip, _ip, _ip, _ip, _ip)
_sig("tbs_read_jacobian_header", _i, _cp, _ip)
_sig("tbs_read_jacobian", _i, _cp, _ip, _dp, _dp, _dp, _dp, _dp)
_sig("tbs_write_jacobian", _i, _cp, _ip, _dp, _dp, _dp, _dp, _dp)
_sig("tbs_validate_mesh", _i, _ip, _ip, _ip, _ip, _ip, _ip, _ip, _ip)
_sig("tbs_gen_structured_header", _i, _i, _i, _i, _ip)
_sig("tbs_gen_structured_mesh", _i, _i, _i, _ip, _ip, _ip, _ip, _ip, _ip, _ip)
_sig("tbs_gen_jacobian", _i, _i, _i, _i, C.c_double, C.c_uint64, _dp, _dp, _dp, _dp, _dp)
_sig("tbs_resize_block_size", _i, _i, _i, _i, _i, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp)
_sig("tbs_create", _i, _i, C.POINTER(_vp))
_sig("tbs_destroy", _i, _vp)
_sig("tbs_set_stream", _i, _vp, _vp)
_sig("tbs_set_mesh", _i, _vp, _i, _i, _i, _i, _i, _i, _ip, _ip, _ip, _ip, _ip, _ip, _ip)
_sig("tbs_set_jacobian", _i, _vp, _dp, _dp, _dp, _dp, _dp)
_sig("tbs_set_jacobian_device", _i, _vp, _vp, _vp, _vp, _vp)
_sig("tbs_set_rhs", _i, _vp, _dp)
_sig("tbs_stage_jacobian", _i, _vp, _dp, _dp, _dp, _dp)
_sig("tbs_set_initial", _i, _vp, _dp)
_sig("tbs_factor", _i, _vp, _i)
_sig("tbs_sweep", _i, _vp, _i, _dp)
_sig("tbs_solve", _i, _vp, C.c_double, _i, _ip, _dp)
_sig("tbs_selftest_timeout", _i, _vp, C.c_longlong)
_sig("tbs_gmres", _i, _vp, _i, _i, C.c_double, _i, _ip, _dp)
_sig("tbs_solve_multi", _i, _vp, _i, _dp, _dp, C.c_double, _i, _ip, _dp, _i)
_sig("tbs_solve_multi_device", _i, _vp, _i, _vp, _vp, C.c_double, _i, _ip, _dp, _i)
_sig("tbs_set_partition_mesh", _i, _vp, _i, _i, _i, _i, _i, _i, _i, _ip, _ip, _ip, _ip, _ip, _ip, _ip)
_sig("tbs_part_start", _i, _vp, _dp)
_sig("tbs_part_solve_du", _i, _vp)
_sig("tbs_part_line_res", _i, _vp, _dp)
_sig("tbs_part_line_vector", _i, _vp, _i, _i, _vp, _i)
_sig("tbs_part_lines_vector", _i, _vp, _i, _i, _ip, _vp, _i)
_sig("tbs_part_owned_norm", _i, _vp, _vp)
_sig("tbs_resid_timer", _i, _vp, C.POINTER(C.c_double), C.POINTER(C.c_longlong), _i)
_sig("tbs_sync", _i, _vp)
_sig("tbs_part_check", _i, _vp, _dp)
_sig("tbs_get_solution", _i, _vp, _dp)
_sig("tbs_get_residual", _i, _vp, _dp)
_sig("tbs_get_update", _i, _vp, _dp)
_sig("tbs_true_residual_norm", _i, _vp, _dp)
_sig("tbs_set_check", _i, _vp, _i)
_sig("tbs_solve_check", _i, _vp, _dp, _ip, _ip)
_sig("tbs_update_values", _i, _vp, _dp, _dp, _dp)
_sig("tbs_memory_allocated", _i, _vp, C.POINTER(C.c_size_t))
_sig("tbs_set_inner_sweeps", _i, _vp, _i)
_sig("tbs_tune_inner", _i, _vp, C.c_double, _i, _ip, _dp)
_sig("tbs_set_inner_schedule", _i, _vp, _i, _i)
_sig("tbs_get_inner_schedule", _i, _vp, _ip, _ip)
_sig("tbs_profile_enable", _i, _vp, _i)
_sig("tbs_profile_reset", _i, _vp)
_sig("tbs_profile_read", _i, _vp, _ip, C.POINTER(_cp), C.POINTER(C.c_longlong), _dp)
_sig("tbs_kernel_bytes", _i, _vp, _cp, _dp)
_sig("tbs_residual_noalloc", _i, _i, _vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _dp)
_sig("tbs_batch_create", _i, C.POINTER(_vp), _i, C.POINTER(_vp))
_sig("tbs_batch_destroy", _i, _vp)
_sig("tbs_batch_last_error", _cp, _vp)
_sig("tbs_batch_size", _i, _vp, _ip)
_sig("tbs_batch_set_stream", _i, _vp, _vp)
_sig("tbs_batch_solve", _i, _vp, C.c_double, _i, _ip, _dp)
_sig("tbs_batch_set_schedule", _i, _vp, _i, _i, _i)
_sig("tbs_batch_get_schedule", _i, _vp, _ip, _ip, _ip)
_sig("tbs_batch_tune", _i, _vp, _ip, _ip, _ip, _dp)
_sig("tbs_batch_set_warps_per_line", _i, _vp, _i)
_sig("tbs_batch_get_warps_per_line", _i, _vp, _ip)
_sig("tbs_batch_set_inner_sweeps", _i, _vp, _i)
_sig("tbs_batch_set_inner_schedule", _i, _vp, _i, _i)
_sig("tbs_batch_tune_inner", _i, _vp, C.c_double, _i, _ip, _ip, _dp)
_sig("tbs_batch_profile_enable", _i, _vp, _i)
_sig("tbs_batch_profile_reset", _i, _vp)
_sig("tbs_batch_profile_read", _i, _vp, _ip, C.POINTER(_cp), C.POINTER(C.c_longlong), _dp)
_sig("tbs_server_create", _i, _i, _i, C.c_size_t, _i, C.POINTER(_vp))
_sig("tbs_server_destroy", _i, _vp)
_sig("tbs_server_last_error", _cp, _vp)
_sig("tbs_server_set_chunk", _i, _vp, _i)
_sig("tbs_server_set_lanes", _i, _vp, C.c_longlong)
_sig("tbs_server_set_lane_splits", _i, _vp, C.POINTER(C.c_longlong), _i)
_sig("tbs_server_add_system", _i, _vp, _i, _i, _i, _i, _i, _i, _ip, _ip, _ip, _ip, _ip, _ip, _ip,
     _dp, _dp, _dp, _ip)
_sig("tbs_server_system_bytes", _i, _vp, _i, _i, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t))
_sig("tbs_server_submit", _i, _vp, _i, _i, _dp, _dp, C.c_double, _i, _dp, _dp, _dp,
     C.POINTER(C.c_longlong))
_sig("tbs_server_poll", _i, _vp, C.c_longlong, _ip)
_sig("tbs_server_wait", _i, _vp, C.c_longlong, _ip, _dp, _dp, _dp)
_sig("tbs_server_stats", _i, _vp, C.POINTER(C.c_longlong), _i)


class TbsError(RuntimeError):
    """A tbs_* call returned a non-zero status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[status {code}] {msg}")
        self.code = code


def last_error(ctx=None) -> str:
    s = lib.tbs_last_error(ctx)
    return s.decode() if s else ""


def check(code: int, ctx=None) -> None:
    if code != TBS_OK:
        raise TbsError(code, last_error(ctx))


def check_server(code: int, srv=None) -> None:
    if code != TBS_OK:
        s = lib.tbs_server_last_error(srv)
        raise TbsError(code, s.decode() if s else "")


def check_batch(code: int, batch=None) -> None:
    if code != TBS_OK:
        s = lib.tbs_batch_last_error(batch)
        raise TbsError(code, s.decode() if s else "")


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)


def dptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def header_functions(path: str = HEADER_PATH) -> list[str]:
    """Names of every function declared in include/triblock.h."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\([^;{]*\)\s*;", text)
    return sorted(set(n for n in names if n not in ("if", "while", "for", "sizeof")))
