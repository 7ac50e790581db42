"""Seeded synthetic inputs in numpy -- TEST INFRASTRUCTURE.

The structured line mesh in the numbering of the reference's data sets
(data/ex05/gpuline.mesh.data.bin is reproduced bit for bit by this rule:
element e = l*K + k, lines in element order, faces numbered by looping e
ascending -- the in-line face (e+1, e) when k+1 < K, then the cross-line
face (e+K, e) when l+1 < L -- and ef per element [S, E, N, W] with negative
boundary codes), and the seeded block values (splitmix64 counter stream, a
uniform double in [-1, 1) per position, drawn in file order jacD, jacO1,
jacO2, rhs; shift * I added to every diagonal block; face blocks scaled by
0.1).  Both are bit-identical to the library's tbs_gen_structured_mesh /
tbs_gen_jacobian (tests/test_generator.py), so bench.py's CPU reference arm
builds the same system without loading the product library.
"""
from __future__ import annotations

from types import SimpleNamespace

import numpy as np

GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_CHUNK = 1 << 22


def splitmix_values(seed: int, start: int, count: int, out: np.ndarray | None = None) -> np.ndarray:
    """U(-1,1) of the counter stream at positions start .. start+count-1."""
    if out is None:
        out = np.empty(count)
    s = np.uint64(seed)
    for c0 in range(0, count, _CHUNK):
        n = np.arange(start + c0, start + min(count, c0 + _CHUNK), dtype=np.uint64)
        with np.errstate(over="ignore"):
            z = s + (n + np.uint64(1)) * GOLDEN
            z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
            z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
            z = z ^ (z >> np.uint64(31))
        out[c0:c0 + n.size] = (z >> np.uint64(11)).astype(np.float64) * 2.0 ** -53 * 2.0 - 1.0
    return out


def structured_mesh(L: int, K: int, nvar: int = 9) -> SimpleNamespace:
    """L lines of K cells, 0-based arrays as after the reference's loader."""
    n = L * K
    e = np.arange(n, dtype=np.int64)
    l, k = e // K, e % K
    hasE = k + 1 < K
    hasN = l + 1 < L
    # faces in element order: E face then N face of each element
    per = hasE.astype(np.int64) + hasN.astype(np.int64)
    first = np.concatenate([[0], np.cumsum(per)[:-1]])
    nf = int(per.sum())
    fidE = np.where(hasE, first, -1)
    fidN = np.where(hasN, first + hasE, -1)
    fc = np.zeros(2 * nf, np.int32)
    fc[2 * fidE[hasE]] = e[hasE] + 1
    fc[2 * fidE[hasE] + 1] = e[hasE]
    fc[2 * fidN[hasN]] = e[hasN] + K
    fc[2 * fidN[hasN] + 1] = e[hasN]
    ef = np.empty((n, 4), np.int64)
    ef[:, 0] = np.where(l > 0, fidN[np.maximum(e - K, 0)], -(k + 1) - 1)
    ef[:, 1] = np.where(hasE, fidE, -(K + l + 1) - 1)
    ef[:, 2] = np.where(hasN, fidN, -(K + L + k + 1) - 1)
    ef[:, 3] = np.where(k > 0, fidE[np.maximum(e - 1, 0)], -(2 * K + L + l + 1) - 1)
    return SimpleNamespace(
        nvar=nvar, nelem=n, nintface=nf, eftot=4 * n, nline=L, nlineelem=n, max_line_nelem=K,
        epoint=(4 * np.arange(n + 1)).astype(np.int32), ef=ef.reshape(-1).astype(np.int32),
        fc=fc, linesize=np.full(L, K, np.int32),
        linepoint=(K * np.arange(L + 1)).astype(np.int32), lines=e.astype(np.int32),
        lineface=ef[:, 3].astype(np.int32))


def jacobian(nv: int, nelem: int, nint: int, shift: float, seed: int):
    """(jacD, jacO1, jacO2, rhs) of the seeded generator."""
    nb = nv * nv
    nD, nO, nR = nb * nelem, nb * nint, nv * nelem
    jacD = splitmix_values(seed, 0, nD)
    d = jacD.reshape(nelem, nv, nv)
    for i in range(nv):
        d[:, i, i] += shift
    O1 = splitmix_values(seed, nD, nO)
    O1 *= 0.1
    O2 = splitmix_values(seed, nD + nO, nO)
    O2 *= 0.1
    rhs = splitmix_values(seed, nD + 2 * nO, nR)
    return jacD, O1, O2, rhs
