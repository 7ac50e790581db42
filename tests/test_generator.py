"""The seeded synthetic Jacobian (tbs_gen_jacobian) against a numpy restatement."""
import numpy as np

from meshes import numpy_jacobian, ragged_mesh
from triblocksolve_b200 import Jacobian, Mesh


def test_generator_bit_exact_against_numpy():
    for (L, K, shift, seed) in [(3, 4, 9.0, 1), (60, 64, 9.0, 1), (7, 5, 4.0, 12345)]:
        m = Mesh.structured(L, K)
        j = Jacobian.generate(m, shift, seed)
        jacD, O1, O2, rhs = numpy_jacobian(9, m.nelem, m.nintface, shift, seed)
        np.testing.assert_array_equal(j.jacD, jacD)
        np.testing.assert_array_equal(j.jacO1, O1)
        np.testing.assert_array_equal(j.jacO2, O2)
        np.testing.assert_array_equal(j.rhs, rhs)
        assert not j.U0.any()


def test_value_distribution():
    m = Mesh.structured(20, 20)
    j = Jacobian.generate(m, 9.0, 7)
    D = j.jacD.reshape(-1, 9, 9)  # [e][col][row]
    diag = np.einsum("eii->ei", D)
    off = D[:, ~np.eye(9, dtype=bool)]
    assert 8.0 <= diag.min() and diag.max() < 10.0
    assert -1.0 <= off.min() and off.max() < 1.0
    assert np.abs(j.jacO1).max() < 0.1 and np.abs(j.jacO2).max() < 0.1
    assert -1.0 <= j.rhs.min() and j.rhs.max() < 1.0
    j2 = Jacobian.generate(m, 9.0, 8)
    assert not np.array_equal(j.rhs, j2.rhs)


def test_generator_other_block_size():
    m = ragged_mesh([4, 2, 5], seed=1, nvar=5)
    j = Jacobian.generate(m, 5.0, 3)
    jacD, O1, O2, rhs = numpy_jacobian(5, m.nelem, m.nintface, 5.0, 3)
    np.testing.assert_array_equal(j.jacD, jacD)
    np.testing.assert_array_equal(j.rhs, rhs)


def test_oracle_synthetic_inputs_equal_the_library():
    """oracle/synthetic.py (what bench.py's CPU reference arm builds its
    system from, without loading the product library) against the library's
    generators, bit for bit."""
    from oracle import synthetic
    for (L, K, nv, shift, seed) in [(1, 1, 9, 9.0, 1), (1, 7, 9, 9.0, 2), (6, 1, 9, 4.0, 3),
                                    (60, 64, 9, 9.0, 1), (7, 5, 5, 5.0, 4)]:
        m = Mesh.structured(L, K, nvar=nv)
        s = synthetic.structured_mesh(L, K, nvar=nv)
        for f in Mesh.FIELDS:
            np.testing.assert_array_equal(getattr(m, f), getattr(s, f), err_msg=f)
        for f in ("nvar", "nelem", "nintface", "eftot", "nline", "nlineelem", "max_line_nelem"):
            assert getattr(m, f) == getattr(s, f), f
        j = Jacobian.generate(m, shift, seed)
        for a, b in zip((j.jacD, j.jacO1, j.jacO2, j.rhs),
                        synthetic.jacobian(nv, m.nelem, m.nintface, shift, seed)):
            np.testing.assert_array_equal(a, b)
