"""triblocksolve_b200 -- B200 (sm_100a) line-implicit Jacobi block solver.

Drop-in for the LIJ path of ackirby88/triblocksolve: the Mesh / Jacobian
classes and their stream-binary files, the block-Thomas factorization and
the LIJ sweep, all on hand-written CUDA behind the C ABI in
include/triblock.h (libtriblock.so).  There is no CPU path.
"""
from ._native import (ALGO_FP64, ALGO_MIXED, ALGO_PIJ, ALGO_REFERENCE, CUDA_MODE, TbsError,  # noqa: F401
                      header_functions, lib)
from .lij import Batch, Jacobian, Mesh, Platform, Solver  # noqa: F401
from .serving import Server  # noqa: F401

__all__ = ["Mesh", "Jacobian", "Platform", "Solver", "Batch", "Server", "TbsError", "ALGO_REFERENCE", "ALGO_FP64",
           "ALGO_MIXED", "ALGO_PIJ", "CUDA_MODE"]
