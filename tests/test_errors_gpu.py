"""Error paths on the device: statuses, never traps; the context stays usable."""
import numpy as np
import pytest

from triblocksolve_b200 import (ALGO_FP64, ALGO_MIXED, ALGO_REFERENCE, Jacobian, Mesh, Platform,
                                Solver, TbsError)
from triblocksolve_b200 import _native as N

pytestmark = pytest.mark.gpu


def test_calls_out_of_order():
    s = Solver(0)
    with pytest.raises(TbsError) as e:
        s.factor(ALGO_FP64)
    assert e.value.code == N.TBS_ERR_STATE
    mesh = Mesh.structured(4, 4)
    s.set_mesh(mesh)
    with pytest.raises(TbsError) as e:
        s.sweep(1)
    assert e.value.code == N.TBS_ERR_STATE
    s.close()


@pytest.mark.parametrize("algo", [ALGO_REFERENCE, ALGO_FP64, ALGO_MIXED])
def test_zero_pivot_reports_numeric_error(algo):
    s = Solver(0)
    mesh = Mesh.structured(4, 6)
    jac = Jacobian.generate(mesh, 9.0, 1)
    bad = jac.jacD.copy()
    bad[81 * 6: 81 * 7] = 0.0  # zero diagonal block of the first cell of line 1 (D' = D)
    s.set_mesh(mesh)
    s.set_jacobian_arrays(bad, jac.jacO1, jac.jacO2, jac.rhs)
    with pytest.raises(TbsError) as e:
        s.factor(algo)
    assert e.value.code == N.TBS_ERR_NUMERIC
    # the context is still usable
    s.set_jacobian(jac)
    s.factor(algo)
    h = s.sweep(3)
    assert np.all(np.isfinite(h)) and h[-1] < h[0]
    s.close()


def test_other_compute_modes_rejected():
    for mode in (0, 1, 3, 4, 5, 6):
        with pytest.raises(TbsError) as e:
            Platform(mode, 0)
        assert e.value.code == N.TBS_ERR_UNSUPPORTED


def test_bad_device_id():
    with pytest.raises(TbsError) as e:
        Platform(2, 4096)
    assert e.value.code == N.TBS_ERR_ARG


def test_block_size_support():
    """FP64 runs at any nvar in 2..16 (general-size kernels); the mixed form
    needs nvar 9 and says so; the reference order takes every size."""
    s = Solver(0)
    from meshes import ragged_mesh
    mesh = ragged_mesh([3, 4], seed=1, nvar=5)
    jac = Jacobian.generate(mesh, 5.0, 1)
    s.set_mesh(mesh)
    s.set_jacobian(jac)
    s.factor(ALGO_FP64)
    with pytest.raises(TbsError) as e:
        s.factor(ALGO_MIXED)
    assert e.value.code == N.TBS_ERR_UNSUPPORTED
    s.factor(ALGO_REFERENCE)
    s.close()


def test_staging_wait_timeout_is_reported_and_recoverable():
    """The bounded wait of every bulk-copy pipeline, made to run out on a
    barrier that nothing completes (no copy is issued): the status comes
    back as an error and the context keeps working."""
    s = Solver(0)
    try:
        mesh = Mesh.structured(6, 8)
        jac = Jacobian.generate(mesh, 9.0, 1)
        s.set_mesh(mesh)
        s.set_jacobian(jac)
        s.factor(ALGO_FP64)
        with pytest.raises(TbsError) as e:
            N.check(N.lib.tbs_selftest_timeout(s.ctx, 1 << 20), s.ctx)  # ~0.5 ms budget
        assert e.value.code == N.TBS_ERR_CUDA
        assert "time budget" in str(e.value)
        n, h = s.solve(1e-12, 100)
        assert h[-1] <= 1e-12 * h[0]
    finally:
        s.close()
