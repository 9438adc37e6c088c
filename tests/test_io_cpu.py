"""CPU checks of the dense file formats (csrc/io.cu through the C ABI): MatrixMarket array text
and the MCNLA binary format, round trips, blocks, the reference's own fixtures when present,
and the error statuses."""
import os

import numpy as np
import pytest

from mcnla_b200 import _lib, io

from oracle.refpath import reference_root

_REF = reference_root()
REF_DATA = os.path.join(_REF, "data") if _REF else None


def test_matrix_market_round_trip_and_blocks(tmp_path):
    rng = np.random.default_rng(1)
    a = rng.standard_normal((37, 53)) * np.logspace(-300, 300, 53)
    a[3, 4] = -0.0
    p = tmp_path / "a.mtx"
    io.save_matrix_market(p, a, comment="a test matrix")
    text = p.read_text().splitlines()
    assert text[0] == "%%MatrixMarket matrix array real general" and text[1] == "% a test matrix"
    assert text[2] == "37 53" and len(text) == 3 + a.size
    assert io.matrix_market_size(p) == (37, 53, 1)
    b = io.load_matrix_market(p)
    assert np.array_equal(b, a) and np.signbit(b[3, 4])          # exact: 17 significant digits
    assert np.array_equal(io.load_matrix_market(p, order="F"), a)
    assert np.array_equal(io.load_matrix_market(p, rows=(5, 11)), a[5:16])          # row block
    assert np.array_equal(io.load_matrix_market(p, cols=(40, 13), order="F"), a[:, 40:])   # column block
    # a column-major source writes the same file
    q = tmp_path / "af.mtx"
    io.save_matrix_market(q, np.asfortranarray(a), comment="a test matrix")
    assert q.read_bytes() == p.read_bytes()


def test_matrix_market_collection(tmp_path):
    rng = np.random.default_rng(2)
    mats = rng.standard_normal((4, 9, 5))           # 4 matrices of 9 x 5
    unfolded = np.concatenate(list(mats), axis=1)    # 9 x 20, matrix k in columns [5k, 5k + 5)
    p = tmp_path / "q.mtx"
    io.save_matrix_market(p, unfolded, nmat=4)
    lines = p.read_text().splitlines()
    assert lines[0] == "%%MatrixMarket 3D array real general" and lines[1] == "9 5 4"
    # file order: matrix after matrix, column-major within each
    assert float(lines[2]) == mats[0, 0, 0] and float(lines[3]) == mats[0, 1, 0]
    assert float(lines[2 + 45]) == mats[1, 0, 0]
    assert io.matrix_market_size(p) == (9, 5, 4)
    assert np.array_equal(io.load_matrix_market(p), unfolded)


@pytest.mark.skipif(not REF_DATA or not os.path.isdir(REF_DATA), reason="the reference's data directory is not here")
def test_reference_fixtures_parse_like_the_golden_conversion():
    golden = np.load(os.path.join(os.path.dirname(__file__), "golden", "mcnla_data.npz"))
    a = io.load_matrix_market(os.path.join(REF_DATA, "a.mtx"))
    assert np.array_equal(a, golden["a"])
    qi = io.load_matrix_market(os.path.join(REF_DATA, "qi.mtx"))
    assert np.array_equal(qi, np.concatenate(list(golden["qi"]), axis=1))
    assert np.array_equal(io.load_matrix_market(os.path.join(REF_DATA, "qb_kn.mtx")), golden["qb_kn"])


def test_binary_round_trip_and_header(tmp_path):
    rng = np.random.default_rng(3)
    a = rng.standard_normal((23, 17))                # row-major m x n: dims {n, m}
    p = tmp_path / "a.bin"
    io.save_binary(p, a, comment="row-major A")
    raw = p.read_bytes()
    assert raw[:23] == b"##MCNLABinaryFileFormat" and raw[31:32] == b"\n"
    assert raw[32:45] == b"# row-major A" and raw[95:96] == b"\n"
    assert raw[96:99] == b"DEN" and raw[104:106] == b"R8" and raw[127:128] == b"\n"
    assert np.frombuffer(raw[128:152], dtype=np.int64).tolist() == [2, 17, 23]
    assert len(raw) == 152 + a.nbytes
    assert io.binary_size(p) == ((17, 23), "R8")
    assert np.array_equal(io.load_binary(p), a)
    assert np.array_equal(io.load_binary(p, first=5, count=7), a[5:12])      # a row block


def test_binary_reads_r4(tmp_path):
    a = np.arange(12, dtype=np.float32).reshape(3, 4) / 7
    head = bytearray(b" " * 128)
    head[:23] = b"##MCNLABinaryFileFormat"
    head[31:32] = b"\n"
    head[32:34] = b"# "
    head[95:96] = b"\n"
    head[96:99] = b"DEN"
    head[104:106] = b"R4"
    head[127:128] = b"\n"
    p = tmp_path / "f.bin"
    p.write_bytes(bytes(head) + np.array([2, 4, 3], dtype=np.int64).tobytes() + a.tobytes())
    assert io.binary_size(p) == ((4, 3), "R4")
    assert np.array_equal(io.load_binary(p), a.astype(np.float64))


def test_error_statuses(tmp_path):
    lib = _lib.load()
    import ctypes
    dims = (ctypes.c_int64 * 3)()
    nd = ctypes.c_int()
    assert lib.mcnla_b200_mm_size(str(tmp_path / "missing.mtx").encode(), dims, ctypes.byref(nd)) == _lib.ERR_IO
    coo = tmp_path / "coo.mtx"
    coo.write_text("%%MatrixMarket matrix coordinate real general\n3 3 1\n1 1 2.0\n")
    assert lib.mcnla_b200_mm_size(str(coo).encode(), dims, ctypes.byref(nd)) == _lib.ERR_IO
    short = tmp_path / "short.mtx"
    short.write_text("%%MatrixMarket matrix array real general\n2 2\n1.0\n2.0\n3.0\n")
    with pytest.raises(RuntimeError):
        io.load_matrix_market(short)
    ok = tmp_path / "ok.mtx"
    io.save_matrix_market(ok, np.eye(3))
    out = np.empty(9)
    assert lib.mcnla_b200_mm_load(str(ok).encode(), 2, 2, 0, 3, out.ctypes.data_as(ctypes.c_void_p), 3,
                                  _lib.ROW_MAJOR) == _lib.ERR_SHAPE
    assert "file" in _lib.status_string(_lib.ERR_IO)
    notbin = tmp_path / "x.bin"
    notbin.write_bytes(b"\0" * 200)
    assert lib.mcnla_b200_binary_size(str(notbin).encode(), dims, ctypes.byref(nd), None) == _lib.ERR_IO


def test_binary_row_reader_fills_row_blocks(tmp_path):
    """The streamed ingest's reader (the reference's loadBinaryRowBlock): rows [row0, row0 + rows)
    of a row-major binary matrix land in a caller's buffer given by address, in any block split."""
    a = np.random.default_rng(3).standard_normal((37, 11))
    p = tmp_path / "a.bin"
    io.save_binary(p, a)
    m, n, read_rows = io.binary_row_reader(p)
    assert (m, n) == (37, 11)
    out = np.empty_like(a)
    for r0, rows in ((0, 5), (5, 16), (21, 16)):
        buf = np.zeros((rows, n))
        read_rows(r0, rows, buf.ctypes.data)
        out[r0:r0 + rows] = buf
    np.testing.assert_array_equal(out, a)
    with pytest.raises(Exception):
        read_rows(30, 10, np.zeros((10, n)).ctypes.data)          # past the last row
