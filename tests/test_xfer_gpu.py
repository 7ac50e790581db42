"""Transfers that keep off the copy engine (csrc/xfer.cu): results read into
pinned host memory by the SMs, and a served request whose right-hand sides
and solutions live in pinned client buffers, must equal the same results
moved by cudaMemcpyAsync into and out of pageable memory, bit for bit.

Stated tolerance: none -- the bytes are copied, not computed.
"""
import numpy as np
import pytest
import torch

from meshes import ragged_mesh
from triblocksolve_b200 import ALGO_FP64, Jacobian, Mesh, Server, Solver

pytestmark = pytest.mark.gpu

TOL = 1e-10


def pinned_like(a):
    t = torch.empty(a.size, dtype=torch.float64, pin_memory=True).numpy().reshape(a.shape)
    t[...] = a
    return t


@pytest.mark.parametrize("mesh_fn", [
    lambda: Mesh.structured(24, 36),
    lambda: ragged_mesh([7, 3, 9, 5, 2], seed=3),          # 26 cells
    lambda: ragged_mesh([5, 1, 7], seed=2, nvar=5),        # nvar 5, 13 cells: not 16-byte sized
])
def test_pinned_and_pageable_read_backs_agree(mesh_fn):
    mesh = mesh_fn()
    jac = Jacobian.generate(mesh, 9.0, 11)
    s = Solver(0)
    try:
        s.set_mesh(mesh)
        s.set_jacobian(jac)
        s.factor(ALGO_FP64)
        n, h = s.solve(TOL, 200)
        assert n > 0
        nv = s.nvar * s.nelem
        for read in (s.solution, s.residual, s.update):
            page = read()
            pin = torch.empty(nv, dtype=torch.float64, pin_memory=True).numpy()
            pin[:] = np.nan
            read(out=pin)
            np.testing.assert_array_equal(pin, page)
    finally:
        s.close()


def test_served_request_with_pinned_client_buffers():
    mesh = Mesh.structured(40, 48)
    jac = Jacobian.generate(mesh, 6.0, 5)
    new_jac = Jacobian.generate(mesh, 5.0, 6)
    rng = np.random.default_rng(9)
    rows = rng.uniform(-1, 1, (3, 9 * mesh.nelem))
    rows2 = rng.uniform(-1, 1, (2, 9 * mesh.nelem))

    def alone(j, rr):
        s = Solver(0)
        try:
            s.set_mesh(mesh)
            s.set_jacobian(j)
            s.factor(ALGO_FP64)
            out = []
            for r in rr:
                s.set_rhs(r)
                n, h = s.solve(TOL, 200)
                out.append((s.solution(), n))
            return out
        finally:
            s.close()

    srv = Server(0, ALGO_FP64, budget_bytes=4 << 30, max_rhs=16, chunk=2)
    try:
        sid = srv.add_system(mesh, jac)
        rhs_pin = pinned_like(rows)
        out_pin = pinned_like(np.full_like(rows, np.nan))
        U, sw, rel, _, _ = srv.submit(sid, rhs_pin, TOL, out=out_pin).wait()
        for k, (u, n) in enumerate(alone(jac, rows)):
            assert sw[k] == n
            np.testing.assert_array_equal(out_pin[k], u)
            np.testing.assert_array_equal(U[k], u)
        # a re-factoring request from pinned Jacobian values (paced upload)
        pj = Jacobian.generate(mesh, 5.0, 6)
        pj.jacD, pj.jacO1, pj.jacO2 = (pinned_like(a) for a in (new_jac.jacD, new_jac.jacO1, new_jac.jacO2))
        out2 = pinned_like(np.full_like(rows2, np.nan))
        U2, sw2, _, _, _ = srv.submit(sid, pinned_like(rows2), TOL, new_jacobian=pj, out=out2).wait()
        for k, (u, n) in enumerate(alone(new_jac, rows2)):
            assert sw2[k] == n
            np.testing.assert_array_equal(out2[k], u)
        assert srv.stats()["refactors"] == 1
    finally:
        srv.close()
