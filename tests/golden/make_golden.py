"""Regenerate the committed fixtures in tests/golden.

Run from the repository root:  python tests/golden/make_golden.py REFERENCE_DIR

REFERENCE_DIR is a checkout of the reference (read only).

Fixtures
  ex05_mesh.json   facts of the reference's only real data file,
                   data/ex05/gpuline.mesh.data.bin (read from REFERENCE_DIR):
                   size, sha256, header and sampled 1-based entries of
                   every array.  The structured generator must reproduce the
                   file bit for bit.
  ex06_sizes.json  sizes and oids of the ex06 Git-LFS pointer files
                   (the data are not in the reference checkout); the size
                   formulas of both layouts must give these byte counts.
  lij_60x64.json   output of the reference's own kernels (OKL translated to
                   C into oracle/_ref by oracle/okl2c.py, built from
                   REFERENCE_DIR here): per-sweep residual norms and
                   solution checksums of the 60x64 / shift 9 / seed 1
                   problem for 20 sweeps.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def ex05(refdir: str) -> dict:
    path = os.path.join(refdir, "data", "ex05", "gpuline.mesh.data.bin")
    raw = open(path, "rb").read()
    a = np.frombuffer(raw, "<i4")
    hdr = [int(v) for v in a[:6]]
    nvar, nelem, nint, eftot, nline, nle = hdr
    sizes = [("epoint", nelem + 1), ("ef", eftot), ("fc", 2 * nint), ("linesize", nline),
             ("linepoint", nline + 1), ("lines", nle), ("lineface", nle)]
    off = 6
    samples = {}
    for name, n in sizes:
        arr = a[off:off + n]
        idx = sorted(set([0, 1, 2, n // 3, n // 2, n - 2, n - 1]))
        samples[name] = {str(i): int(arr[i]) for i in idx if 0 <= i < n}
        off += n
    return {"file": "data/ex05/gpuline.mesh.data.bin", "bytes": len(raw),
            "sha256": hashlib.sha256(raw).hexdigest(), "header": hdr,
            "samples_1based": samples, "structured": {"L": 60, "K": 64}}


def ex06(refdir: str) -> dict:
    out = {}
    for name in ("gpuline.jacobian.data.bin", "gpuline.mesh.data.bin"):
        txt = open(os.path.join(refdir, "data", "ex06", name)).read().split("\n")
        kv = dict(line.split(" ", 1) for line in txt if " " in line)
        out[name] = {"oid": kv["oid"], "size": int(kv["size"])}
    out["cells"] = 138240
    out["structured"] = {"L": 360, "K": 384}
    return out


def lij_golden(refdir: str) -> dict:
    import oracle
    from triblocksolve_b200 import Jacobian, Mesh
    if not oracle.ref_available():
        oracle.build_ref(refdir)
    mesh = Mesh.structured(60, 64)
    jac = Jacobian.generate(mesh, 9.0, 1)
    r = oracle.ref_lij(mesh, jac.jacD, jac.jacO1, jac.jacO2, jac.rhs, 20, threads=1)
    U = r["U"]
    return {"problem": {"L": 60, "K": 64, "shift": 9.0, "seed": 1, "sweeps": 20},
            "hist": [float(v) for v in r["hist"]],
            "U_sum": float(U.sum()), "U_sumsq": float((U * U).sum()),
            "U_first": [float(v) for v in U[:9]], "U_last": [float(v) for v in U[-9:]],
            "note": "the reference's own kernels (lineLU_v2.okl, linesmoothLU_TriBlock_v3.okl, "
                    "linesmoothLU_v5.okl translated to C by oracle/okl2c.py), one thread"}


def main():
    import argparse
    ap = argparse.ArgumentParser(description="regenerate tests/golden fixtures")
    ap.add_argument("reference_dir", help="a checkout of the reference (read only)")
    refdir = ap.parse_args().reference_dir
    if not os.path.isdir(os.path.join(refdir, "src", "okl")):
        ap.error(f"{refdir} is not a checkout of the reference")
    with open(os.path.join(HERE, "ex05_mesh.json"), "w") as f:
        json.dump(ex05(refdir), f, indent=1)
    with open(os.path.join(HERE, "ex06_sizes.json"), "w") as f:
        json.dump(ex06(refdir), f, indent=1)
    with open(os.path.join(HERE, "lij_60x64.json"), "w") as f:
        json.dump(lij_golden(refdir), f, indent=1)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
