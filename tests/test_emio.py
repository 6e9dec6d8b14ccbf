"""EM-format I/O (IOfun/tom_emread.m:153-176, IOfun/tom_emwrite.m:94-150):
the 512-byte header layout, both byte orders, and the data types a reader
meets.  Host-only: runs without a GPU."""
import numpy as np
import pytest

from conftest import needs_library

pytestmark = needs_library


def _header(magic, dims, comment=b""):
    h = bytearray(512)
    h[0:4] = bytes(magic)
    be = magic[0] in (0, 3, 5)
    h[4:16] = np.asarray(dims, ">i4" if be else "<i4").tobytes()
    h[16:16 + len(comment)] = comment
    return bytes(h)


def test_write_layout_and_round_trip(tmp_path):
    from tom_b200 import tom_emread, tom_emwrite
    rng = np.random.default_rng(3)
    v = np.asfortranarray(rng.standard_normal((7, 5, 3)).astype(np.float32))
    p = tmp_path / "a.em"
    tom_emwrite(p, v, "hello")
    raw = p.read_bytes()
    assert len(raw) == 512 + 4 * v.size
    assert raw[:4] == bytes([6, 0, 0, 5])
    assert np.array_equal(np.frombuffer(raw[4:16], "<i4"), [7, 5, 3])
    assert raw[16:21] == b"hello"
    assert np.array_equal(np.frombuffer(raw[512:], "<f4"), v.ravel(order="F"))
    r = tom_emread(p)
    assert r["Header"]["Size"] == (7, 5, 3)
    assert np.array_equal(r["Value"], v)


@pytest.mark.parametrize("order,code", [("<", 6), (">", 3), (">", 0)])
@pytest.mark.parametrize("dtype,tcode", [("i2", 2), ("i4", 4), ("f4", 5), ("f8", 9), ("u1", 1)])
def test_read_types_and_byte_orders(tmp_path, order, code, dtype, tcode):
    from tom_b200 import tom_emread
    rng = np.random.default_rng(4)
    v = (rng.standard_normal((4, 3, 2)) * 50).astype(dtype if dtype == "u1" else order + dtype)
    if dtype == "u1":
        v = np.abs(v).astype("u1")
    p = tmp_path / "b.em"
    p.write_bytes(_header([code, 0, 0, tcode], v.shape) + np.asfortranarray(v).tobytes(order="F"))
    r = tom_emread(p)
    assert np.array_equal(r["Value"], v.astype(np.float32))


def test_truncated_file_rejected(tmp_path):
    from tom_b200 import tom_emread, TomGpuError
    p = tmp_path / "c.em"
    p.write_bytes(_header([6, 0, 0, 5], (10, 10, 10)) + b"\0" * 100)
    with pytest.raises(TomGpuError):
        tom_emread(p)
