"""Build steps for the native code (run by __graft_entry__.build()).

``build_all()`` compiles libtriblock.so and triblock.exe for sm_100a with
nvcc (triblocksolve_b200/csrc/Makefile) and the CPU oracle used by the tests
(oracle/Makefile).  Both are plain make invocations; outputs stay in-tree.
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


def build_all() -> None:
    build_library()
    build_oracle()


if __name__ == "__main__":
    build_all()
