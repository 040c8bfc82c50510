"""Result files in the reference's <HDR> format (no GPU needed).

Bars: the nd_Ek header the library writes is the reference's own byte for
byte (its Si_Bulk.nd_Ek header with the count changed), the reader parses the
reference's file, and appending keeps earlier records and updates the count.
"""
import ctypes as C

import numpy as np
import pytest

from nemo3d_b200 import build as nb
from nemo3d_b200 import nd_files


@pytest.fixture(scope="module")
def lib():
    nb.build()
    L = C.CDLL(nb.LIB)
    L.tbgpu_write_eigenvalues.argtypes = [C.c_char_p, C.c_char, C.c_void_p, C.c_int, C.c_void_p]
    return L


def _ref(golden):
    return bytes(golden["si_bulk_nd_ek_head"])


def test_reader_parses_reference_file(golden, tmp_path):
    head = _ref(golden)
    p = tmp_path / "ref.nd_Ek"
    p.write_bytes(head)
    hdr, rec = nd_files.read(str(p))
    assert hdr["format"] == "{real kx, real ky, real kz, real E}"
    assert hdr["dims"] == [6400] and hdr["dim_labels"] == ["# number of eigenvalues"]
    assert len(rec) == 16 and np.all(np.isfinite(rec["E"]))


def test_header_matches_reference_bytes(lib, golden, tmp_path):
    head = _ref(golden)
    end = head.index(b"<\\HDR>") + 6
    recs = np.frombuffer(head[end:], np.float64).reshape(16, 4)
    p = str(tmp_path / "ours.nd_Ek").encode()
    assert lib.tbgpu_write_eigenvalues(p, b"i", None, 0, None) == 0
    k = np.ascontiguousarray(recs[0, :3])
    E = np.ascontiguousarray(recs[:, 3])
    assert np.all(recs[:, :3] == recs[0, :3])  # one k point in these records
    assert lib.tbgpu_write_eigenvalues(p, b"a", k.ctypes.data, 16, E.ctypes.data) == 0
    ours = open(p, "rb").read()
    want = head[:end].replace(b"= 6400       #", b"= 16         #") + head[end:]
    assert ours == want


def test_append_keeps_records(lib, tmp_path):
    p = str(tmp_path / "x.nd_Ek").encode()
    assert lib.tbgpu_write_eigenvalues(p, b"i", None, 0, None) == 0
    k1 = np.array([0.1, 0.0, 0.0])
    k2 = np.array([0.2, 0.0, 0.0])
    e1 = np.array([-1.5, 0.25, 1.75])
    e2 = np.array([2.0, 3.0, 4.0, 5.0, 6.0])
    assert lib.tbgpu_write_eigenvalues(p, b"a", k1.ctypes.data, 3, e1.ctypes.data) == 0
    assert lib.tbgpu_write_eigenvalues(p, b"a", k2.ctypes.data, 5, e2.ctypes.data) == 0
    kE = nd_files.read_eigenvalues(p.decode())
    assert kE.shape == (8, 4)
    np.testing.assert_array_equal(kE[:, 3], np.concatenate([e1, e2]))
    np.testing.assert_array_equal(kE[:3, 0], 0.1)
    np.testing.assert_array_equal(kE[3:, 0], 0.2)


def test_bad_arguments(lib, tmp_path):
    p = str(tmp_path / "y.nd_Ek").encode()
    assert lib.tbgpu_write_eigenvalues(p, b"x", None, 0, None) == -1
    assert lib.tbgpu_write_eigenvalues(p, b"a", None, 2, None) == -1
    bad = tmp_path / "bad.nd_Ek"
    bad.write_bytes(b"not a header file")
    e = np.array([1.0])
    assert lib.tbgpu_write_eigenvalues(str(bad).encode(), b"a", None, 1, e.ctypes.data) == -1
