"""triblock.exe on the GPU: the reference's entry point with the forms this
build adds (point-implicit sweep, several right-hand sides, GMRES, other
block sizes), each run to completion with its report."""
import json
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "triblocksolve_b200", "bin", "triblock.exe")


def run(*args):
    r = subprocess.run([EXE, "2", "0", *args], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def last_json(out):
    return json.loads([l for l in out.splitlines() if l.startswith("{")][-1])


def test_fixed_sweeps_reference_default():
    out = run("9", "--gen", "20", "24", "9", "1", "--json")
    assert last_json(out)["sweeps"] == 30


def test_point_implicit():
    out = run("9", "--gen", "20", "24", "9", "1", "--algo", "pij", "--tol", "1e-10", "--json")
    j = last_json(out)
    assert j["true_rel_resid"] <= 1.0000001e-10


def test_several_right_hand_sides():
    out = run("9", "--gen", "20", "24", "9", "1", "--nrhs", "5", "--tol", "1e-10")
    assert sum(1 for l in out.splitlines() if l.strip().startswith("rhs ")) == 5


def test_gmres():
    out = run("9", "--gen", "20", "24", "3", "1", "--gmres", "20", "--tol", "1e-10", "--json")
    assert "GMRES(20)" in out
    assert last_json(out)["true_rel_resid"] <= 1.0000001e-10


@pytest.mark.parametrize("nv", ["5", "12"])
def test_other_block_sizes(nv):
    out = run(nv, "--gen", "20", "24", "12", "1", "--tol", "1e-10", "--json")
    j = last_json(out)
    assert j["true_rel_resid"] <= 1.0000001e-10


def test_options_need_tolerance():
    r = subprocess.run([EXE, "2", "0", "9", "--gen", "4", "4", "9", "1", "--nrhs", "2"],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
