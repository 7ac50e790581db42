"""Mesh / Jacobian file formats (src/F90/read_mesh_data.F90, read_jacobian_data.F90)."""
import ctypes as C
import hashlib
import json
import os

import numpy as np
import pytest

from triblocksolve_b200 import Jacobian, Mesh, TbsError
from triblocksolve_b200 import _native as N

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_structured_generator_reproduces_ex05(tmp_path):
    gold = json.load(open(os.path.join(GOLD, "ex05_mesh.json")))
    m = Mesh.structured(60, 64)
    assert list(m.header) == gold["header"]
    p = str(tmp_path / "m.bin")
    m.toFile(p)
    raw = open(p, "rb").read()
    assert len(raw) == gold["bytes"]
    assert hashlib.sha256(raw).hexdigest() == gold["sha256"]
    # sampled 1-based entries, array by array
    a = np.frombuffer(raw, "<i4")
    off = 6
    for name, n in [("epoint", m.nelem + 1), ("ef", m.eftot), ("fc", 2 * m.nintface),
                    ("linesize", m.nline), ("linepoint", m.nline + 1), ("lines", m.nlineelem),
                    ("lineface", m.nlineelem)]:
        for i, v in gold["samples_1based"][name].items():
            assert a[off + int(i)] == v, (name, i)
        off += n


def test_read_converts_to_zero_based(tmp_path):
    m = Mesh.structured(5, 7)
    p = str(tmp_path / "m.bin")
    m.toFile(p)
    raw = np.fromfile(p, "<i4")
    assert raw[6] == 1  # epoint[0] on disk
    r = Mesh.from_file(p)
    for f in Mesh.FIELDS:
        np.testing.assert_array_equal(getattr(r, f), getattr(m, f))
    assert r.epoint[0] == 0 and r.linepoint[0] == 0 and r.lines[0] == 0
    assert r.max_line_nelem == 7


def test_fortran_reader_entry_points(tmp_path, monkeypatch):
    """read_mesh_data_ / read_jacobian_data_ keep the Fortran bind(C) signatures."""
    m = Mesh.structured(4, 6)
    j = Jacobian.generate(m, 9.0, 3)
    monkeypatch.chdir(tmp_path)
    m.toFile("gpuline.mesh.data.bin")
    j.toFile("gpuline.jacobian.data.bin")
    ints = [C.c_int(v) for v in m.header]
    arr = {f: np.zeros_like(getattr(m, f)) for f in Mesh.FIELDS}
    N.lib.read_mesh_data_.restype = None
    N.lib.read_mesh_data_(*[C.byref(v) for v in ints], N.iptr(arr["epoint"]), N.iptr(arr["ef"]),
                          N.iptr(arr["fc"]), N.iptr(arr["lines"]), N.iptr(arr["linesize"]),
                          N.iptr(arr["linepoint"]), N.iptr(arr["lineface"]))
    for f in Mesh.FIELDS:
        np.testing.assert_array_equal(arr[f], getattr(m, f))
    jd = {k: np.zeros_like(getattr(j, k)) for k in ("jacD", "jacO1", "jacO2", "rhs", "U0")}
    jints = [C.c_int(m.nvar), C.c_int(m.nelem), C.c_int(m.nintface)]
    N.lib.read_jacobian_data_.restype = None
    N.lib.read_jacobian_data_(*[C.byref(v) for v in jints], *[N.dptr(jd[k]) for k in
                                                             ("jacD", "jacO1", "jacO2", "rhs", "U0")])
    for k, v in jd.items():
        np.testing.assert_array_equal(v, getattr(j, k))


def test_jacobian_round_trip_and_layout(tmp_path):
    m = Mesh.structured(3, 5)
    j = Jacobian.generate(m, 4.0, 11)
    p = str(tmp_path / "j.bin")
    j.toFile(p)
    raw = open(p, "rb").read()
    assert np.frombuffer(raw[:12], "<i4").tolist() == [9, m.nelem, m.nintface]
    # FP64 data start at byte 12 (unaligned), in file order jacD, O1, O2, rhs, U0
    body = np.frombuffer(raw[12:], "<f8")
    nD, nO = 81 * m.nelem, 81 * m.nintface
    np.testing.assert_array_equal(body[:nD], j.jacD)
    np.testing.assert_array_equal(body[nD:nD + nO], j.jacO1)
    np.testing.assert_array_equal(body[nD + 2 * nO:nD + 2 * nO + 9 * m.nelem], j.rhs)
    r = Jacobian()
    r.fromFile(m.nlineelem, p)
    for k in ("jacD", "jacO1", "jacO2", "rhs", "U0"):
        np.testing.assert_array_equal(getattr(r, k), getattr(j, k))
    assert r.A.size == 81 * m.nlineelem and r.DinvC.size == 81 * m.nelem


def test_size_formulas_match_ex06_pointers(tmp_path):
    """The ex06 Jacobian is only an LFS pointer; its byte count fixes the layout."""
    gold = json.load(open(os.path.join(GOLD, "ex06_sizes.json")))
    m = Mesh.structured(360, 384)
    assert m.nelem == gold["cells"]
    want = gold["gpuline.jacobian.data.bin"]["size"]
    p = str(tmp_path / "ex06_like.bin")
    with open(p, "wb") as f:
        f.write(np.array([9, m.nelem, m.nintface], "<i4").tobytes())
    os.truncate(p, want)  # sparse file of exactly the pointer's size
    hdr = np.zeros(3, np.int32)
    assert N.lib.tbs_read_jacobian_header(p.encode(), N.iptr(hdr)) == N.TBS_OK
    os.truncate(p, want - 8)
    assert N.lib.tbs_read_jacobian_header(p.encode(), N.iptr(hdr)) == N.TBS_ERR_FORMAT
    # the real ex06 mesh lists 5,544 more bytes of faces than the structured rule
    mp = str(tmp_path / "m.bin")
    m.toFile(mp)
    assert gold["gpuline.mesh.data.bin"]["size"] - os.path.getsize(mp) == 5544


def test_missing_and_truncated_files(tmp_path):
    with pytest.raises(TbsError) as e:
        Mesh.from_file(str(tmp_path / "nope.bin"))
    assert e.value.code == N.TBS_ERR_IO
    m = Mesh.structured(4, 4)
    p = str(tmp_path / "m.bin")
    m.toFile(p)
    data = open(p, "rb").read()
    open(p, "wb").write(data[:-4])
    with pytest.raises(TbsError) as e:
        Mesh.from_file(p)
    assert e.value.code == N.TBS_ERR_FORMAT
    open(p, "wb").write(data[:10])
    with pytest.raises(TbsError) as e:
        Mesh.from_file(p)
    assert e.value.code == N.TBS_ERR_IO
    bad = np.frombuffer(data, "<i4").copy()
    bad[1] = -5
    bad.tofile(p)
    with pytest.raises(TbsError) as e:
        Mesh.from_file(p)
    assert e.value.code == N.TBS_ERR_FORMAT


def test_reader_rejects_caller_size_mismatch(tmp_path):
    m = Mesh.structured(4, 4)
    p = str(tmp_path / "m.bin")
    m.toFile(p)
    hdr = m.header.copy()
    hdr[1] += 1
    arrs = [np.zeros(10000, np.int32) for _ in range(7)]
    rc = N.lib.tbs_read_mesh(p.encode(), N.iptr(hdr), *[N.iptr(a) for a in arrs])
    assert rc == N.TBS_ERR_FORMAT


def _mesh_arrays(m):
    return {f: getattr(m, f).copy() for f in Mesh.FIELDS}


@pytest.mark.parametrize("breakage", ["lines_dup", "lineface_wrong", "fc_range", "linepoint",
                                      "nlineelem", "empty_line", "ef_range"])
def test_validation_rejects_broken_meshes(breakage):
    m = Mesh.structured(4, 5)
    a = _mesh_arrays(m)
    nv = m.nvar
    if breakage == "lines_dup":
        a["lines"][3] = a["lines"][4]
    elif breakage == "lineface_wrong":
        a["lineface"][2] = a["lineface"][7]
    elif breakage == "fc_range":
        a["fc"][5] = m.nelem
    elif breakage == "linepoint":
        a["linepoint"][2] += 1
    elif breakage == "nlineelem":
        a["lines"] = a["lines"][:-1]
        a["lineface"] = a["lineface"][:-1]
        a["linesize"][-1] -= 1
        a["linepoint"][-1] -= 1
    elif breakage == "empty_line":
        a["linesize"][0] = 0
    elif breakage == "ef_range":
        a["ef"][3] = m.nintface
    mm = Mesh.from_arrays(nv, **a)
    with pytest.raises(TbsError) as e:
        mm.validate()
    assert e.value.code == N.TBS_ERR_FORMAT


def test_structured_and_ragged_meshes_validate():
    from meshes import ragged_mesh
    Mesh.structured(60, 64).validate()
    Mesh.structured(1, 1).validate()
    Mesh.structured(1, 9).validate()
    Mesh.structured(9, 1).validate()
    ragged_mesh([5, 1, 7, 3, 3, 8], seed=4).validate()
