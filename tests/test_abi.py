"""The C ABI library: loads, exports every declared symbol, fails loudly
without a device (no CPU fallback).  No compute calls."""
import ctypes as C
import os
import subprocess

import pytest

from triblocksolve_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_every_header_function_is_exported():
    names = N.header_functions()
    assert "tbs_create" in names and "read_mesh_data_" in names and len(names) >= 30
    missing = [n for n in names if not hasattr(N.lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", N.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert set(names) <= exported


def test_version_string():
    assert b"sm_100a" in N.lib.tbs_version()


def test_null_context_is_an_argument_error():
    assert N.lib.tbs_factor(None, 1) == N.TBS_ERR_ARG
    assert N.lib.tbs_sweep(None, 1, None) == N.TBS_ERR_ARG
    assert N.lib.tbs_destroy(None) == N.TBS_OK
    assert N.lib.tbs_part_start(None, None) == N.TBS_ERR_ARG
    assert N.lib.tbs_part_solve_du(None) == N.TBS_ERR_ARG
    assert N.lib.tbs_part_line_res(None, None) == N.TBS_ERR_ARG
    assert N.lib.tbs_part_line_vector(None, N.VEC_UPDATE, 0, None, 0) == N.TBS_ERR_ARG
    assert N.lib.tbs_create(0, None) == N.TBS_ERR_ARG


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_no_device_fails_loudly():
    h = C.c_void_p()
    rc = N.lib.tbs_create(0, C.byref(h))
    assert rc == N.TBS_ERR_CUDA
    assert "no CPU path" in N.last_error()
    assert not h.value


def test_cli_help_and_mode_check():
    exe = os.path.join(ROOT, "triblocksolve_b200", "bin", "triblock.exe")
    r = subprocess.run([exe, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "compute_mode" in r.stdout
    r = subprocess.run([exe, "0", "0", "9", "--gen", "2", "2", "9", "1"], capture_output=True,
                       text=True)
    assert r.returncode == 1 and "mode 2" in r.stderr
    r = subprocess.run([exe, "2", "0", "9", "--bogus"], capture_output=True, text=True)
    assert r.returncode == 2
