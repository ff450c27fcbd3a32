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
