"""psphray-format snapshots (psg_snapshot_write / psg_snapshot_read): a
round trip through the library, and the same file read by the reference's
own reader (src/reader.c, src/reader-psphray.c, built into
oracle/_ref/libpsphray_reader.so when the reference is present)."""
import ctypes as C
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_READER = os.path.join(ROOT, "oracle", "_ref", "libpsphray_reader.so")


def _arrays(n, seed=0):
    rng = np.random.default_rng(seed)
    return {"pos": rng.random((n, 3)).astype(np.float32), "id": rng.integers(0, 1 << 40, n),
            "mass": rng.random(n).astype(np.float32), "ie": rng.random(n).astype(np.float32),
            "rho": rng.random(n).astype(np.float32), "ye": rng.random(n).astype(np.float32),
            "xHI": rng.random(n).astype(np.float32), "sml": rng.random(n).astype(np.float32),
            "xHeI": rng.random(n).astype(np.float32), "xHeII": rng.random(n).astype(np.float32),
            "gammaHI": rng.random(n).astype(np.float32), "lasthit": rng.integers(0, 10000, n),
            "hits": rng.integers(0, 1000, n).astype(np.int32)}


CONSTS = dict(time=0.125, redshift=7.0, boxsize=4752.0, OmegaM=0.26, OmegaL=0.74, OmegaB=0.044, h=0.72)


def test_round_trip(tmp_path):
    from psphray_b200 import api
    a = _arrays(1000)
    src = np.array([[1.0, 2.0, 3.0], [4.0, 5.0, 6.0]], np.float32)
    ng = np.array([1e-3, 2e-3])
    path = str(tmp_path / "snap_000")
    api.write_snapshot(path, 1000, a, src_pos=src, ngammas=ng, **CONSTS)
    r = api.read_snapshot(path)
    assert r["ngas"] == 1000 and r["nsrc"] == 2
    for k in CONSTS:
        assert r[k] == CONSTS[k]
    for k, v in a.items():
        assert np.array_equal(r[k], v), k
    assert np.array_equal(r["src_pos"], src) and np.array_equal(r["ngammas"], ng)
    # the block layout: header + 13 gas blocks + ngammas + spec, each with two size markers
    item = {"pos": 12, "id": 8, "mass": 4, "lasthit": 8}
    gas = sum(item.get(k, 4) * (1002 if k in ("pos", "id", "mass") else 1000) + 8 for k in a)
    assert os.path.getsize(path) == 256 + 8 + gas + 2 * (2 * 8 + 8)


def test_missing_arrays_are_zeros(tmp_path):
    from psphray_b200 import api
    path = str(tmp_path / "snap_zero")
    api.write_snapshot(path, 10, {"xHI": np.ones(10, np.float32)}, **CONSTS)
    r = api.read_snapshot(path)
    assert np.all(r["xHI"] == 1.0) and np.all(r["mass"] == 0.0) and np.all(r["lasthit"] == 0)


@pytest.mark.skipif(not os.path.exists(REF_READER), reason="the reference's reader was not built here")
def test_reference_reader_reads_our_file(tmp_path):
    from psphray_b200 import api
    n = 777
    a = _arrays(n, seed=3)
    src = np.array([[0.5, 0.25, 0.125]], np.float32)
    ng = np.array([3.5e-2])
    path = str(tmp_path / "snap_ref")
    api.write_snapshot(path, n, a, src_pos=src, ngammas=ng, **CONSTS)
    L = C.CDLL(REF_READER)
    f = L.refrd_read
    f.restype = C.c_int
    ngas, nsrc = C.c_size_t(0), C.c_size_t(0)
    consts = np.zeros(7)
    nulls = [None] * 15
    f(path.encode(), C.byref(ngas), C.byref(nsrc), consts.ctypes.data_as(C.c_void_p), *nulls)
    assert ngas.value == n and nsrc.value == 1
    assert list(consts) == [CONSTS[k] for k in ("time", "redshift", "boxsize", "OmegaM", "OmegaL", "OmegaB", "h")]
    out = {k: np.zeros_like(v) for k, v in a.items()}
    sp, ngr = np.zeros((1, 3), np.float32), np.zeros(1)
    order = ["pos", "id", "mass", "ie", "rho", "ye", "xHI", "sml", "xHeI", "xHeII", "gammaHI", "lasthit", "hits"]
    f(path.encode(), C.byref(ngas), C.byref(nsrc), consts.ctypes.data_as(C.c_void_p),
      *[C.c_void_p(out[k].ctypes.data) for k in order], C.c_void_p(sp.ctypes.data), C.c_void_p(ngr.ctypes.data))
    for k in order:
        assert np.array_equal(out[k], a[k]), k
    assert np.array_equal(sp, src) and np.array_equal(ngr, ng)
