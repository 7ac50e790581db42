"""Build steps for the native code (run by __graft_entry__.build()).

``build_all()`` compiles libtriblock.so and triblock.exe for sm_100a with
nvcc (triblocksolve_b200/csrc/Makefile) and the CPU oracle used by the tests
(oracle/Makefile).  Where a checkout of the reference exists (the directory
in $TBS_REFERENCE_DIR, default /root/reference), it also translates and
compiles the reference's own kernels into oracle/_ref (``make ref``), the
checker the oracle is pinned to.  All are plain make invocations; outputs
stay in-tree.
"""
from __future__ import annotations

import os
import subprocess

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
REPO_DIR = os.path.dirname(PKG_DIR)


def _make(path: str, jobs: int = 8) -> None:
    subprocess.run(["make", "-j", str(jobs), "-C", path], check=True)


def build_library() -> str:
    _make(os.path.join(PKG_DIR, "csrc"))
    return os.path.join(PKG_DIR, "lib", "libtriblock.so")


def build_oracle() -> str:
    _make(os.path.join(REPO_DIR, "oracle"))
    return os.path.join(REPO_DIR, "oracle", "_build", "liboracle.so")


def build_reference_checker() -> str | None:
    ref = os.environ.get("TBS_REFERENCE_DIR", "/root/reference")
    if not os.path.isdir(os.path.join(ref, "src", "okl")):
        return None
    subprocess.run(["make", "-C", os.path.join(REPO_DIR, "oracle"), "ref", f"REFERENCE={ref}"],
                   check=True)
    return os.path.join(REPO_DIR, "oracle", "_ref", "libokl_ref.so")


def build_all() -> None:
    build_library()
    build_oracle()
    build_reference_checker()


if __name__ == "__main__":
    build_all()
