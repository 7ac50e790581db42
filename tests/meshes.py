"""Test meshes and numpy restatements used by the test-suite.

``ragged_mesh`` builds line meshes the structured generator never produces:
lines of different lengths, element ids permuted, faces listed in random
order with random (e1, e2) orientation, boundary markers interleaved in
``ef``, lines listed in shuffled order.  ``splitmix_values`` restates the
seeded value generator of tbs_gen_jacobian in numpy.
"""
from __future__ import annotations

import numpy as np

from triblocksolve_b200 import Jacobian, Mesh

GOLDEN = 0x9E3779B97F4A7C15
M64 = (1 << 64) - 1


def splitmix_values(seed: int, start: int, count: int) -> np.ndarray:
    """U(-1,1) of stream positions start..start+count-1 (numpy uint64 arithmetic)."""
    n = np.arange(start, start + count, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + (n + np.uint64(1)) * np.uint64(GOLDEN)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * 2.0 ** -53 * 2.0 - 1.0


def numpy_jacobian(nv, nelem, nint, shift, seed):
    nb = nv * nv
    nD, nO, nR = nb * nelem, nb * nint, nv * nelem
    jacD = splitmix_values(seed, 0, nD)
    idx = np.arange(nD)
    diag = (idx % nv) == ((idx // nv) % nv)
    jacD[diag] += shift
    O1 = 0.1 * splitmix_values(seed, nD, nO)
    O2 = 0.1 * splitmix_values(seed, nD + nO, nO)
    rhs = splitmix_values(seed, nD + 2 * nO, nR)
    return jacD, O1, O2, rhs


def ragged_mesh(lens, seed=0, nvar=9, permute=True) -> Mesh:
    rng = np.random.default_rng(seed)
    L = len(lens)
    cells = [(l, k) for l in range(L) for k in range(lens[l])]
    index = {c: i for i, c in enumerate(cells)}
    N = len(cells)
    elem = rng.permutation(N) if permute else np.arange(N)
    faces = []
    for (l, k) in cells:
        if k + 1 < lens[l]:
            faces.append((index[(l, k)], index[(l, k + 1)]))
        if l + 1 < L and k < lens[l + 1]:
            faces.append((index[(l, k)], index[(l + 1, k)]))
    order = rng.permutation(len(faces)) if permute else np.arange(len(faces))
    fc = np.zeros(2 * len(faces), np.int32)
    face_id = {}
    for fid, j in enumerate(order):
        a, b = faces[j]
        ea, eb = int(elem[a]), int(elem[b])
        if permute and rng.random() < 0.5:
            ea, eb = eb, ea
        fc[2 * fid], fc[2 * fid + 1] = ea, eb
        face_id[frozenset((a, b))] = fid
    per_elem = [[] for _ in range(N)]
    for key, fid in face_id.items():
        for c in key:
            per_elem[int(elem[c])].append(fid)
    nb_count = 0
    for e in range(N):
        while len(per_elem[e]) < 4:
            nb_count += 1
            per_elem[e].append(-1 - nb_count)
        if permute:
            rng.shuffle(per_elem[e])
    epoint = np.zeros(N + 1, np.int32)
    for e in range(N):
        epoint[e + 1] = epoint[e] + len(per_elem[e])
    ef = np.array([f for e in range(N) for f in per_elem[e]], np.int32)
    line_order = rng.permutation(L) if permute else np.arange(L)
    lines, linesize, lineface = [], [], []
    for l in line_order:
        linesize.append(lens[l])
        for k in range(lens[l]):
            lines.append(int(elem[index[(l, k)]]))
            if k == 0:
                lineface.append(-7)
            else:
                lineface.append(face_id[frozenset((index[(l, k - 1)], index[(l, k)]))])
    linepoint = np.concatenate([[0], np.cumsum(linesize)]).astype(np.int32)
    m = Mesh.from_arrays(nvar, epoint=epoint, ef=ef, fc=fc, linesize=np.array(linesize, np.int32),
                         linepoint=linepoint, lines=np.array(lines, np.int32),
                         lineface=np.array(lineface, np.int32))
    m.validate()
    return m


def problem(mesh: Mesh, shift=9.0, seed=1) -> Jacobian:
    return Jacobian.generate(mesh, shift, seed)


def point_mesh(mesh: Mesh) -> Mesh:
    """The same cells and faces with every cell its own line (the line sweep
    on it is the point-implicit Jacobi sweep)."""
    n = mesh.nelem
    return Mesh.from_arrays(mesh.nvar, epoint=mesh.epoint, ef=mesh.ef, fc=mesh.fc,
                            linesize=np.ones(n, np.int32), linepoint=np.arange(n + 1, dtype=np.int32),
                            lines=np.arange(n, dtype=np.int32), lineface=np.full(n, -1, np.int32))
