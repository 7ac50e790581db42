"""The hand restatement (oracle/lij_oracle.c) pinned to the reference's own
code: the OKL kernels of lineLU_v2.okl, linesmoothLU_TriBlock_v3.okl and
linesmoothLU_v5.okl and the Jacobian methods of Jacobian.cxx, translated
mechanically to C by oracle/okl2c.py into oracle/_ref and driven in
src/main.cxx:180-229 order (oracle/ref_driver.c).

Bar: bit-identical factors, packed lower blocks, and U, R, dU after every
sweep, on the structured meshes of the benchmark configs, ragged meshes with
permuted numbering, a single line, one-cell lines, and block sizes 2, 5, 9,
12 and 16 (the span of the general-size kernels).

oracle/_ref is built by `make -C oracle ref REFERENCE=<reference checkout>`
(the package build does it where the checkout exists); without it these
tests skip.
"""
import numpy as np
import pytest

import oracle
from meshes import point_mesh, ragged_mesh
from triblocksolve_b200 import Jacobian, Mesh

pytestmark = pytest.mark.skipif(not oracle.ref_available(),
                                reason="oracle/_ref not built (make -C oracle ref "
                                       "REFERENCE=<reference checkout>)")

CASES = {
    "60x64": (lambda: Mesh.structured(60, 64), 9.0, 20),
    "60x64_shift4": (lambda: Mesh.structured(60, 64), 4.0, 12),
    "ragged": (lambda: ragged_mesh([5, 1, 7, 3, 3, 8, 13, 2, 9], seed=4), 9.0, 10),
    "ragged_permuted_2": (lambda: ragged_mesh([17, 4, 4, 30, 1, 6], seed=11), 6.0, 10),
    "single_line": (lambda: Mesh.structured(1, 37), 9.0, 8),
    "single_cells": (lambda: Mesh.structured(6, 1), 9.0, 8),
    "one_cell_lines": (lambda: point_mesh(Mesh.structured(8, 10)), 9.0, 8),
    "nvar5": (lambda: Mesh.structured(12, 16, nvar=5), 9.0, 10),
    "nvar5_ragged": (lambda: ragged_mesh([4, 6, 2, 5], seed=2, nvar=5), 5.0, 8),
    "nvar2": (lambda: Mesh.structured(10, 12, nvar=2), 4.0, 8),
    "nvar12_ragged": (lambda: ragged_mesh([3, 7, 1, 5], seed=5, nvar=12), 12.0, 6),
    "nvar16": (lambda: Mesh.structured(6, 9, nvar=16), 16.0, 6),
}


@pytest.mark.parametrize("case", list(CASES))
def test_restatement_equals_reference_kernels(case):
    make, shift, iters = CASES[case]
    mesh = make()
    jac = Jacobian.generate(mesh, shift, 3)
    ref = oracle.ref_lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, iters, per_sweep=True,
                         want_factors=True)
    b = oracle.Baseline(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, 2)
    np.testing.assert_array_equal(b.DLU, ref["DLU"])
    np.testing.assert_array_equal(b.DinvC, ref["DinvC"])
    np.testing.assert_array_equal(b.A, ref["A"][: b.A.size])
    for p in range(iters):
        b.sweeps(1)
        np.testing.assert_array_equal(b.U, ref["U_all"][p], err_msg=f"U after sweep {p + 1}")
        np.testing.assert_array_equal(b.R, ref["R_all"][p], err_msg=f"R after sweep {p + 1}")
        np.testing.assert_array_equal(b.dU, ref["dU_all"][p], err_msg=f"dU after sweep {p + 1}")
    o = oracle.lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, iters)
    np.testing.assert_array_equal(o["hist"], ref["hist"])


def test_reference_kernels_thread_count_independent():
    mesh = Mesh.structured(30, 40)
    jac = Jacobian.generate(mesh, 4.0, 5)
    a = oracle.ref_lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, 6, threads=1)
    b = oracle.ref_lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, 6, threads=4)
    for k in ("U", "R", "dU", "hist"):
        np.testing.assert_array_equal(a[k], b[k])


def test_true_residual_equals_reference_line_res():
    mesh = ragged_mesh([9, 2, 11, 5], seed=7)
    jac = Jacobian.generate(mesh, 9.0, 8)
    U = np.random.default_rng(1).uniform(-1, 1, jac.rhs.size)
    np.testing.assert_array_equal(
        oracle.true_residual(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, U),
        oracle.ref_true_residual(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, U))


@pytest.mark.parametrize("nv_new", [4, 5, 7, 9, 10, 12, 16])
def test_resize_block_size_equals_reference(nv_new):
    mesh = Mesh.structured(5, 6)
    jac = Jacobian.generate(mesh, 9.0, 9)
    U0 = np.random.default_rng(2).uniform(-1, 1, jac.rhs.size)
    args = (9, nv_new, mesh.nelem, mesh.nintface, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, U0)
    for a, b in zip(oracle.resize_block_size(*args), oracle.ref_resize_block_size(*args)):
        np.testing.assert_array_equal(a, b)


def test_resized_system_sweeps_equal():
    """The reference's resize followed by its sweeps, against the restatement's."""
    mesh9 = Mesh.structured(10, 12)
    jac = Jacobian.generate(mesh9, 9.0, 4)
    U0 = np.zeros(jac.rhs.size)
    D, O1, O2, rhs, _ = oracle.ref_resize_block_size(9, 5, mesh9.nelem, mesh9.nintface, jac.jacD,
                                                     jac.jacO1, jac.jacO2, jac.rhs, U0)
    mesh5 = Mesh.structured(10, 12, nvar=5)
    a = oracle.ref_lij(mesh5, D, O1, O2, rhs, 6)
    b = oracle.lij(mesh5, D, O1, O2, rhs, 6)
    for k in ("U", "R", "dU", "hist"):
        np.testing.assert_array_equal(a[k], b[k])
