"""The two launch forms of the line solve give bit-identical results.

The single-system line solve (FP64, and the FP32 inner sweeps of the mixed
form) has a one-warp form and a warp-specialised form (a copy warp beside
the chain warp), picked by how many lines share an SM; the test meshes are
small, so by default they always get the warp-specialised form.  Here the
same solves run in two processes with each form forced (TBS_THOMAS_WS=0 /
1, read once per process) and must agree bit for bit; so must the
several-right-hand-side solve run beside them.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import triblocksolve_b200 as tbs
mesh = tbs.Mesh.structured(20, 24)
jac = tbs.Jacobian.generate(mesh, 4.0, 3)
s = tbs.Solver(0)
s.set_mesh(mesh)
s.set_jacobian(jac)
s.factor(tbs.ALGO_FP64)
n, h = s.solve(1e-10, 100)
U = s.solution()
rows = np.stack([jac.rhs, -jac.rhs, np.linspace(-1.0, 1.0, jac.rhs.size)])
Um, sw, hm = s.solve_multi(rows, 1e-10, 100)
s.factor(tbs.ALGO_MIXED)
n2, h2 = s.solve(1e-10, 100)
U2 = s.solution()
s.close()
np.savez(sys.argv[2], n=n, h=h, U=U, Um=Um, sw=sw, hm=np.concatenate(hm), n2=n2, h2=h2, U2=U2)
"""


def _run(tmp_path, form):
    out = str(tmp_path / f"form{form}.npz")
    env = dict(os.environ, TBS_THOMAS_WS=str(form))
    subprocess.run([sys.executable, "-c", SCRIPT, ROOT, out], env=env, check=True, timeout=300)
    return np.load(out)


def test_one_warp_and_warp_specialised_forms_agree(tmp_path):
    a, b = _run(tmp_path, 0), _run(tmp_path, 1)
    for k in a.files:
        assert np.array_equal(a[k], b[k]), k
    assert int(a["n"]) > 1 and np.all(a["sw"] > 1)

