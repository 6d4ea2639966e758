"""STORE ... BINARY: a result written as segment files by the device segment writer.

The stored table must read back (in a later script, through the catalog) as the same rows
the oracle gives for the result, and every segment file must be byte for byte the host
writer's image of its column (the host writer is pinned to the reference's own files in
test_golden.py). Headers follow writeHeader (cm.cu:1251-1263): total rows, segments,
largest segment, largest payload."""
import ctypes
import os

import numpy as np
import pytest

import alenka_b200 as ab

from . import _oracle
from .test_gpu_parity import _read

pytestmark = pytest.mark.gpu

SELECT = ("LF := FILTER lineitem BY l_shipdate < 19950101 AND l_quantity > 10;\n"
          "R := SELECT l_orderkey AS ok, l_quantity AS q, l_extendedprice AS p, l_discount AS dc, "
          "l_shipdate AS sd FROM LF;\n")
COLS = ["ok", "q", "p", "dc", "sd"]


@pytest.fixture(scope="module")
def flat(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("store_bin"))
    ab.gen_lineitem_flat(d, 300_000, 100_000, 17)
    _oracle.execute(d, SELECT + "STORE R INTO 'want.txt' USING ('|');\n")
    return d


def _rows(text):
    return [ln.split("|")[:len(COLS)] for ln in text.decode().splitlines()]


def _col_values(rows, k):
    return np.array([int(r[k].replace(".", "")) for r in rows], dtype=np.int64)


def _host_image(vals, delta):
    L = ab.lib()
    L.alk_encode_segment.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_void_p,
                                     ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
    v = np.ascontiguousarray(vals, dtype=np.int64)
    out = ctypes.create_string_buffer(24 + 8 * len(v) + 64)
    ln = ctypes.c_size_t()
    assert L.alk_encode_segment(v.ctypes.data, len(v), delta, out, len(out), ctypes.byref(ln)) == 0
    return out.raw[:ln.value]


def _header(path):
    b = open(path, "rb").read()
    return (int.from_bytes(b[0:8], "little"), int.from_bytes(b[8:12], "little"),
            int.from_bytes(b[12:16], "little"), int.from_bytes(b[16:20], "little"))


def _read_back(d, table, out):
    with ab.Session(d) as s:
        s.execute(f"S := SELECT ok AS ok, q AS q, p AS p, dc AS dc, sd AS sd FROM {table};\n"
                  f"STORE S INTO '{out}' USING ('|');\n")
    return _read(os.path.join(d, out))


@pytest.mark.parametrize("delta", [False, True])
def test_store_binary_reads_back_and_matches_host_writer(flat, delta):
    d = flat
    table = "saved_d" if delta else "saved"
    with ab.Session(d, delta=delta) as s:
        s.execute(SELECT + f"STORE R INTO '{table}' BINARY;\n")
    want = _read(os.path.join(d, "want.txt"))
    assert _read_back(d, table, f"{table}_back.txt") == want
    rows = _rows(want)
    for k, c in enumerate(COLS):
        vals = _col_values(rows, k)
        img = open(os.path.join(d, f"{table}.{c}.0"), "rb").read()
        assert img == _host_image(vals, 1 if delta else 0), c
        assert _header(os.path.join(d, f"{table}.{c}.header")) == (len(rows), 1, len(rows),
                                                                    int.from_bytes(img[0:4], "little"))
    if delta:  # the generated orderkeys are in order: that column is written FOR-delta
        img = open(os.path.join(d, f"{table}.ok.0"), "rb").read()
        assert int.from_bytes(img[20:24], "little") == 1


def test_store_binary_append_and_limit(flat):
    d = flat
    with ab.Session(d) as s:
        s.execute(SELECT + "STORE R INTO 'app' BINARY;\n")
        s.execute(SELECT + "STORE R INTO 'app' APPEND LIMIT 1000 BINARY;\n")
    want = _read(os.path.join(d, "want.txt"))
    lines = want.split(b"\n")
    assert _read_back(d, "app", "app_back.txt") == want + b"\n" + b"\n".join(lines[:1000])
    n = len(lines)
    total, segs, max_recs, _ = _header(os.path.join(d, "app.q.header"))
    assert (total, segs, max_recs) == (n + 1000, 2, n)
    rows = _rows(b"\n".join(lines[:1000]))
    assert open(os.path.join(d, "app.p.1"), "rb").read() == _host_image(_col_values(rows, 2), 0)


def test_store_binary_refusals_and_empty(flat):
    d = flat
    with ab.Session(d) as s:
        with pytest.raises(ab.AlenkaError) as e:
            s.execute("LF := FILTER lineitem BY l_quantity > 10;\n"
                      "R := SELECT l_returnflag AS f, l_quantity AS q FROM LF;\n"
                      "STORE R INTO 'chars' BINARY;\n")
        assert "char columns" in str(e.value)
        with pytest.raises(ab.AlenkaError) as e:
            s.execute(SELECT + "STORE R INTO 'sorted' BINARY SORT SEGMENTS BY ok;\n")
        assert "SORT SEGMENTS" in str(e.value)
        s.execute("LF := FILTER lineitem BY l_shipdate < 19000101;\n"
                  "R := SELECT l_orderkey AS ok, l_quantity AS q FROM LF;\n"
                  "STORE R INTO 'nothing' BINARY;\n")
    # an empty select result has no columns (as in the reference), so nothing is written
    assert not os.path.exists(os.path.join(d, "nothing.ok.header"))
    assert not os.path.exists(os.path.join(d, "nothing.ok.0"))
