"""linalg::io binary containers (the reference's wire format,
include/linalg/io.h:66-94, 425-533) through the C ABI, on the host: byte
layout, round trips, and the reference's own data tables when present."""
import os
import struct

import numpy as np
import pytest

MAT_F64 = 0x616d6464      # 'm','a' | 'd' dense | 'd' double
VEC_F64 = 0x65766464      # 'v','e' | 'd' dense | 'd' double


def test_matrix_and_vector_bytes(ibk, tmp_path):
    ibk.build()
    p = str(tmp_path / "obj.bin")
    x = np.arange(12, dtype=np.float64).reshape(4, 3) * 0.5    # 4 points x 3 dims
    v = np.array([1.0, -2.0, 3.5])
    ibk.io_write(p, [x, v, 2.25])
    raw = open(p, "rb").read()
    assert struct.unpack("<4i", raw[:16]) == (MAT_F64, 4, 3, 12)
    # column-major: the x[d*n + p] layout of the reference's point matrices
    assert np.array_equal(np.frombuffer(raw[16:16 + 96], dtype="<f8"), x.T.reshape(-1))
    o = 16 + 96
    assert struct.unpack("<4i", raw[o:o + 16]) == (VEC_F64, 3, 1, 3)
    assert np.array_equal(np.frombuffer(raw[o + 16:o + 40], dtype="<f8"), v)
    assert struct.unpack("<d", raw[o + 40:o + 48])[0] == 2.25
    assert len(raw) == o + 48
    back = ibk.io_read(p, count=2)
    assert np.array_equal(back[0], x) and np.array_equal(back[1], v)


def test_reads_fp32_containers_and_rejects_garbage(ibk, tmp_path):
    ibk.build()
    p = str(tmp_path / "f32.bin")
    vals = np.array([[1.5, 2.5], [3.25, -4.0]], dtype="<f4")
    with open(p, "wb") as f:
        f.write(struct.pack("<4i", 0x616d6473, 2, 2, 4))
        f.write(vals.T.tobytes())
    (m,) = ibk.io_read(p)
    assert m.dtype == np.float64 and np.array_equal(m, vals.astype(np.float64))
    bad = str(tmp_path / "bad.bin")
    with open(bad, "wb") as f:
        f.write(struct.pack("<4i", 0x12345678, 1, 1, 1) + b"\0" * 8)
    with pytest.raises(ibk.IbkError):
        ibk.io_read(bad)
    short = str(tmp_path / "short.bin")
    with open(short, "wb") as f:
        f.write(struct.pack("<4i", VEC_F64, 4, 1, 4) + b"\0" * 8)
    with pytest.raises(ibk.IbkError):
        ibk.io_read(short)


MAT_SPARSE_F64 = 0x616d7364   # 'm','a' | 's' sparse | 'd' double
VEC_SPARSE_F64 = 0x65767364


def test_sparse_containers_bytes_and_round_trip(ibk, tmp_path):
    """io.h:432-470: (rows, cols, nonzeros), a matrix's CSR row starts (rows +
    1 ints), the indices, then the values."""
    import scipy.sparse as sp
    ibk.build()
    p = str(tmp_path / "sparse.bin")
    m = sp.csr_matrix(np.array([[0.0, 1.5, 0.0, -2.0], [0.0, 0.0, 0.0, 0.0], [3.0, 0.0, 4.25, 0.0]]))
    ibk.io_write_sparse(p, m)
    ibk.io_write_sparse(p, (6, [1, 4], [0.5, -7.0]), append=True)
    ibk.io_write(str(tmp_path / "dense.bin"), [np.ones(2)])
    raw = open(p, "rb").read()
    assert struct.unpack("<4i", raw[:16]) == (MAT_SPARSE_F64, 3, 4, 4)
    assert struct.unpack("<4i", raw[16:32]) == (0, 2, 2, 4)                 # row starts
    assert struct.unpack("<4i", raw[32:48]) == (1, 3, 0, 2)                 # column indices
    assert struct.unpack("<4d", raw[48:80]) == (1.5, -2.0, 3.0, 4.25)
    assert struct.unpack("<4i", raw[80:96]) == (VEC_SPARSE_F64, 6, 1, 2)
    assert struct.unpack("<2i", raw[96:104]) == (1, 4)
    assert struct.unpack("<2d", raw[104:120]) == (0.5, -7.0)
    assert len(raw) == 120
    back_m, back_v = ibk.io_read(p)
    assert (back_m != m).nnz == 0 and back_m.shape == (3, 4)
    assert back_v[0] == 6 and list(back_v[1]) == [1, 4] and list(back_v[2]) == [0.5, -7.0]


def test_sparse_edge_cases_and_mixed_files(ibk, tmp_path):
    import scipy.sparse as sp
    ibk.build()
    # an empty matrix writes no row starts
    p = str(tmp_path / "empty.bin")
    ibk.io_write_sparse(p, sp.csr_matrix((0, 5)))
    assert open(p, "rb").read() == struct.pack("<4i", MAT_SPARSE_F64, 0, 5, 0)
    (e,) = ibk.io_read(p)
    assert e.shape == (0, 5) and e.nnz == 0
    # FP32 values are read as FP64
    q = str(tmp_path / "f32.bin")
    with open(q, "wb") as f:
        f.write(struct.pack("<4i", 0x616d7373, 2, 2, 2) + struct.pack("<3i", 0, 1, 2) + struct.pack("<2i", 1, 0))
        f.write(struct.pack("<2f", 1.25, -0.5))
    (m,) = ibk.io_read(q)
    assert np.array_equal(m.toarray(), np.array([[0.0, 1.25], [-0.5, 0.0]]))
    # dense and sparse containers in one file
    r = str(tmp_path / "mixed.bin")
    rng = np.random.default_rng(1)
    dense = rng.normal(size=(5, 3))
    sparse = sp.random(40, 30, density=0.1, random_state=2, format="csr")
    ibk.io_write(r, [dense])
    ibk.io_write_sparse(r, sparse, append=True)
    ibk.io_write(r + ".v", [rng.normal(size=4)])
    with open(r, "ab") as f:
        f.write(open(r + ".v", "rb").read())
    a, b, c = ibk.io_read(r)
    assert np.array_equal(a, dense) and (b != sparse).nnz == 0 and c.shape == (4,)


# the reference's data tables, where its tree is available (IBK_REFERENCE_ROOT)
REF_DATA = os.path.join(os.environ.get("IBK_REFERENCE_ROOT", ""), "data")


@pytest.mark.skipif(not os.environ.get("IBK_REFERENCE_ROOT") or not os.path.isdir(REF_DATA),
                    reason="reference data tables not present (set IBK_REFERENCE_ROOT)")
@pytest.mark.parametrize("name,n", [("rbc.864.bin", 864), ("plt.386.bin", 386)])
def test_reads_the_reference_data_tables(ibk, name, n):
    """The reference's sample-site tables (data/*.bin: n x 2 matrices of
    surface parameters) read back with the expected shape and finite values."""
    ibk.build()
    (m,) = ibk.io_read(os.path.join(REF_DATA, name), count=1)
    assert m.shape == (n, 2) and np.all(np.isfinite(m))
