"""CPU: instance and bias file formats of the reference (jmat.hpp:57-178: SNOWGPU1, SCAJINT8, SCABIAS1, G-set text)
round-trip, and host-side fault injection -- truncated files, wrong magic, trailing bytes, asymmetric couplings,
out-of-range bias, bad or duplicate G-set edges -- is refused with an error, as the reference's loaders refuse it;
the C ABI refuses invalid couplings and tables with ANC_EINVAL before any device work."""
import ctypes as C
import os

import numpy as np
import pytest

from anechoic_b200 import _lib
from anechoic_b200 import instances as I


def _roundtrip(tmp_path, inst, writer, reader):
    p = str(tmp_path / "f.bin")
    writer(inst, p)
    back = reader(p)
    assert back.n == inst.n and np.array_equal(back.to_dense(), inst.to_dense())
    return p


def test_roundtrips(tmp_path):
    _roundtrip(tmp_path, I.complete_pm1(300, 4), I.write_snowgpu1, I.read_snowgpu1)
    _roundtrip(tmp_path, I.random_kbit(200, 4, 5, pzero=0.3), I.write_jint8, I.read_jint8)
    g = I.random_graph(150, 600, True, 6)
    p = str(tmp_path / "g.txt")
    I.write_gset(g, p)
    assert np.array_equal(I.read_gset(p).to_dense(), g.to_dense())
    b = np.arange(-40, 40, dtype=np.int32)
    I.write_bias(b, str(tmp_path / "b.bin"))
    assert np.array_equal(I.read_bias(str(tmp_path / "b.bin"), 80), b)


def _corrupt(path, data):
    with open(path, "wb") as f:
        f.write(data)


def test_truncated_and_wrong_magic_files(tmp_path):
    inst = I.random_kbit(64, 2, 1, pzero=0.2)
    p = str(tmp_path / "j.bin")
    I.write_jint8(inst, p)
    raw = open(p, "rb").read()
    for bad, msg in ((raw[:-1], "short"), (raw + b"\0", "trailing"), (b"SCAJINT9" + raw[8:], "header")):
        _corrupt(p, bad)
        with pytest.raises(ValueError, match=msg):
            I.read_jint8(p)
    g = str(tmp_path / "g.bin")
    I.write_snowgpu1(I.complete_pm1(64, 2), g)
    raw = open(g, "rb").read()
    _corrupt(g, raw[:100])
    with pytest.raises(ValueError, match="short"):
        I.read_snowgpu1(g)
    _corrupt(g, b"SNOWGPU0" + raw[8:])
    with pytest.raises(ValueError, match="header"):
        I.read_snowgpu1(g)
    bp = str(tmp_path / "b.bin")
    I.write_bias(np.zeros(64, np.int32), bp)
    with pytest.raises(ValueError, match="length"):
        I.read_bias(bp, 65)
    I.write_bias(np.full(64, 40000, np.int32), bp)
    with pytest.raises(ValueError, match="32767"):
        I.read_bias(bp, 64)


def test_asymmetric_couplings_and_bad_gset(tmp_path):
    d = I.random_kbit(32, 2, 2, pzero=0.2).dense.copy()
    d[0, 5], d[5, 0] = 1, -1
    p = str(tmp_path / "j.bin")
    I.write_jint8(I.Instance(n=32, dense=d), p)
    with pytest.raises(ValueError, match="symmetric"):
        I.read_jint8(p)
    gp = str(tmp_path / "g.txt")
    for text, msg in (("4 2\n1 2 1\n2 2 1\n", "edge"), ("4 2\n1 2 1\n2 1 1\n", "duplicate"),
                      ("4 2\n1 2 1\n3 4 500\n", "int8"), ("4 2\n1 2 1\n3 4\n", None)):
        open(gp, "w").write(text)
        with pytest.raises(ValueError, match=msg):
            I.read_gset(gp)


def test_abi_refuses_invalid_input_without_device_work():
    L = _lib.load()
    bad = np.zeros((4, 4), np.int8)
    bad[0, 1] = 1
    h = C.c_void_p()
    assert L.anc_instance_create(bad.ctypes.data, 4, 0, None, C.byref(h)) == _lib.ANC_EINVAL
    assert b"symmetric" in L.anc_last_error()
    ok = np.zeros((4, 4), np.int8)
    assert L.anc_instance_create(ok.ctypes.data, 4, 3, None, C.byref(h)) == _lib.ANC_EINVAL   # kbits 3
    f = np.array([0, 4], np.int32)   # 4T must be positive
    z = np.zeros(2, np.int32)
    kc = np.zeros(2, np.int64)
    assert L.anc_tables_create(f.ctypes.data, z.ctypes.data, kc.ctypes.data, z.ctypes.data, 2, C.byref(h)) == \
        _lib.ANC_EINVAL
