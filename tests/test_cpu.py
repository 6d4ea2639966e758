"""CPU-only tests: the C ABI library loads and exports every declared symbol, the front
end emits the reference's postfix queues, the segment codec and MurmurHash64A of the
oracle agree with independent Python restatements, and the oracle's operator results
agree with a numpy recomputation of the same query on the decoded columns."""
import ctypes
import glob
import os
import re
import struct

import numpy as np
import pytest

import alenka_b200 as ab
from alenka_b200 import workloads as wl

from . import _oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    hdr = open(os.path.join(ROOT, "include", "alenka_b200.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    names = set(re.findall(r"^\s*(?:int|void|const char\*|alk_stream)\s+\*?(\w+)\s*\(", hdr, flags=re.M))
    assert {"alenkaInit", "alenkaExecute", "alenkaClose", "execute_file", "alk_scan_filter",
            "alk_groupby_hash", "alk_join_probe", "alk_decode_segment"} <= names
    L = ab.lib()
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing


def _dump(script):
    L = ab.lib()
    L.alk_parse_dump.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]
    buf = ctypes.create_string_buffer(1 << 16)
    rc = L.alk_parse_dump(script.encode(), buf, len(buf))
    return rc, buf.value.decode()


def test_parser_postfix_matches_grammar_actions():
    rc, d = _dump(wl.three_way_script(1))
    assert rc == 0
    lines = d.splitlines()
    # FILTER: NAME NUMBER CMP with the comparison code in op_nums (fl.l:121-127)
    assert lines[0].startswith("FILTER s=OFI f=orders")
    assert lines[1] == " type: NAME NUMBER CMP"
    assert lines[3].split()[-1] == "1"  # '<'
    # string literal and '==' (code 4)
    assert " type: NAME STRING CMP" in d and " nums: 4" in d
    # join: innermost JOIN recorded first (bison.y:259-275), ON columns follow the select list
    j = d[d.index("JOIN s=OLC"):]
    assert "join: CF/I OFI/I sel=5 tabs=2 and: 0=0 1=0" in j
    assert "value: o_orderkey o_orderkey o_orderdate o_orderdate o_shippriority o_shippriority l_extendedprice price " \
           "l_discount discount l_orderkey o_orderkey o_custkey c_custkey" in j
    # SUM(price*(1-discount)): NAME NUMBER NAME MINUS MUL SUM, then the group columns
    s = d[d.index("SELECT s=F"):]
    assert "NAME NUMBER NAME MINUS MUL SUM emit sel_name" in s
    assert s.split("\n")[0].endswith("grp=3 sep=")
    # ORDER: NAME DESC / NAME ASC become (column, direction) pairs (operators.cu:240-250)
    o = d[d.index("ORDER s=RES"):]
    assert " type: sum_revenue orderdate1" in o and " value: DESC ASC" in o
    # STORE LIMIT goes to op_nums (emit_limit)
    assert "STORE s=RES f=q3.txt grp=0 sep=|\n type:\n value:\n nums: 10" in d


def test_parser_decimal_and_precedence():
    rc, d = _dump("A := FILTER t BY a < 1.25 AND b == 3 OR c >= -0.5;")
    assert rc == 0
    assert " type: NAME NUMBER CMP NAME NUMBER CMP AND NAME NUMBER CMP OR" in d
    assert " nums: 125 1 3 4 -5 6" in d
    assert " prec: 2 0 1" in d
    rc, d = _dump("A := FILTER t BY a = 1;")  # '=' is the join operator, not a comparison
    assert " type: NAME NUMBER JOIN" in d
    rc, _ = _dump("A := FILTER t BY ;")
    assert rc == 7


def _py_decode(path):
    """pfor_decompress (compress.cu:180-267) restated in Python."""
    raw = open(path, "rb").read()
    cnt, lower, upper, comp = struct.unpack_from("<Iqq I", raw, 0)
    tail = raw[24 + cnt:]
    _, rec, bits, orig_lower, fit, start = struct.unpack_from("<IIIqIq", tail, 0)
    payload = raw[24:24 + cnt]
    if comp == 0:
        dt = {8: np.uint8, 16: np.uint16, 32: np.uint32, 64: np.uint64}[bits]
        v = np.frombuffer(payload, dtype=dt, count=rec).astype(np.uint64)
        return (v + np.uint64(orig_lower & 0xFFFFFFFFFFFFFFFF)).astype(np.int64)
    words = np.frombuffer(payload, dtype=np.uint64)
    i = np.arange(rec, dtype=np.uint64)
    w = words[(i // fit).astype(np.int64)]
    sh = np.uint64(64 - bits) - (i % np.uint64(fit)) * np.uint64(bits)
    mask = np.uint64((1 << bits) - 1) if bits < 64 else np.uint64(0xFFFFFFFFFFFFFFFF)
    d = ((w >> sh) & mask) + np.uint64(orig_lower & 0xFFFFFFFFFFFFFFFF)
    d[0] = np.uint64(start & 0xFFFFFFFFFFFFFFFF)
    return np.cumsum(d, dtype=np.uint64).astype(np.int64)


@pytest.mark.parametrize("delta", [False, True])
def test_oracle_codec_matches_python(tmp_path, delta):
    ab.gen_lineitem_flat(str(tmp_path), 50_000, 20_000, 3, delta=delta)
    files = [f for f in glob.glob(str(tmp_path / "lineitem.*.*")) if re.search(r"\.\d+(\.idx)?$", f)]
    assert len(files) == 7 * 3
    kinds = set()
    for f in files:
        a = _oracle.decode_file(f)
        b = _py_decode(f)
        assert np.array_equal(a, b), f
        kinds.add(struct.unpack_from("<I", open(f, "rb").read(), 20)[0])
    if delta:
        assert 1 in kinds  # l_orderkey is sorted -> FOR-delta


def _py_murmur(data: bytes, seed=100):
    m = 0xc6a4a7935bd1e995
    M = (1 << 64) - 1
    h = (seed ^ (len(data) * m)) & M
    n8 = len(data) // 8
    for i in range(n8):
        k = struct.unpack_from("<Q", data, 8 * i)[0]
        k = (k * m) & M
        k ^= k >> 47
        k = (k * m) & M
        h ^= k
        h = (h * m) & M
    t = data[8 * n8:]
    if t:
        for j in reversed(range(len(t))):
            h ^= t[j] << (8 * j)
        h = (h * m) & M
    h ^= h >> 47
    h = (h * m) & M
    h ^= h >> 47
    return h


def test_murmur_matches_python():
    rng = np.random.default_rng(0)
    for n in list(range(0, 33)) + [50, 100]:
        data = rng.integers(0, 256, size=n, dtype=np.uint8).tobytes()
        assert _oracle.murmur64a(data) == _py_murmur(data)


def test_oracle_flat_query_matches_numpy(tmp_path):
    d = str(tmp_path)
    ab.gen_lineitem_flat(d, 120_000, 50_000, 9)
    _oracle.execute(d, wl.flat_script(9))
    cols = {}
    for c in ["l_quantity", "l_extendedprice", "l_discount", "l_shipdate", "l_orderkey"]:
        cols[c] = np.concatenate([_py_decode(os.path.join(d, f"lineitem.{c}.{g}")) for g in range(3)])
    for c in ["l_returnflag", "l_linestatus"]:
        codes = np.concatenate([_py_decode(os.path.join(d, f"lineitem.{c}.{g}.idx")) for g in range(3)])
        dic = open(os.path.join(d, f"lineitem.{c}"), "rb").read()
        cols[c] = np.array([dic[x:x + 1].decode() for x in codes])
    keep = cols["l_shipdate"] < wl.flat_cutoff(9)
    want = {}
    for f in "ANR":
        for s in "FO":
            m = keep & (cols["l_returnflag"] == f) & (cols["l_linestatus"] == s)
            rev = int(np.sum(cols["l_extendedprice"][m] * (100 - cols["l_discount"][m])))
            want[(f, s)] = (int(cols["l_quantity"][m].sum()), int(cols["l_extendedprice"][m].sum()), rev, int(m.sum()))
    got = {}
    for line in open(os.path.join(d, "q1.txt")).read().split("\n"):
        f, s, q, p, r, c, _ = line.split("|")
        got[(f, s)] = (int(q), int(p.replace(".", "")), int(r.replace(".", "")), int(c))
    assert got == want


def test_oracle_three_way_matches_numpy(tmp_path):
    d = str(tmp_path)
    wl.make_three_way(d, scale=0.003, seg_rows=100_000, seed=8)
    script = wl.three_way_script(8, limit=0)
    _oracle.execute(d, script)

    def col(t, c, segs):
        return np.concatenate([_py_decode(os.path.join(d, f"{t}.{c}.{g}")) for g in range(segs)])
    date, seg = wl.three_way_params(8)
    cust = np.concatenate([_py_decode(os.path.join(d, f"customer.c_mktsegment.{g}.idx")) for g in range(1)])
    dic = open(os.path.join(d, "customer.c_mktsegment"), "rb").read()
    names = [dic[i:i + 10].rstrip(b"\0").decode() for i in range(0, len(dic), 10)]
    ck = col("customer", "c_custkey", 1)
    good_c = set(ck[np.array([names[x] == seg for x in cust])].tolist())
    ok, oc, od = col("orders", "o_orderkey", 1), col("orders", "o_custkey", 1), col("orders", "o_orderdate", 1)
    mo = (od < date) & np.array([x in good_c for x in oc.tolist()])
    odate = dict(zip(ok[mo].tolist(), od[mo].tolist()))
    nli = sum(1 for _ in glob.glob(os.path.join(d, "lineitem.l_orderkey.*"))) - 1
    lk, ls = col("lineitem", "l_orderkey", nli), col("lineitem", "l_shipdate", nli)
    lp, ldc = col("lineitem", "l_extendedprice", nli), col("lineitem", "l_discount", nli)
    agg = {}
    # OLC aliases l_extendedprice AS price and l_discount AS discount; a join's alias keeps
    # the decimal flag but not the scale (operators.cu:877-906), so both compute at scale
    # 0: price in cents times (1 - discount in hundredths), printed without a point
    for k, s, p, dd in zip(lk.tolist(), ls.tolist(), lp.tolist(), ldc.tolist()):
        if s > date and k in odate:
            r, c = agg.get(k, (0, 0))
            agg[k] = (r + p * (1 - dd), c + 1)
    rows = sorted(agg.items(), key=lambda kv: (-kv[1][0], odate[kv[0]], kv[0]))
    got = open(os.path.join(d, "q3.txt")).read().split("\n")
    assert len(got) == len(rows)
    for line, (k, (r, c)) in zip(got, rows):
        f = line.split("|")
        assert int(f[0]) == k and int(f[1]) == odate[k] and int(f[3]) == r and int(f[4]) == c


def _replica_rank(rank, world, port, q):
    import torch
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # each replica reports its own time; the job's time is the slowest replica's
        ms = bench.max_over_ranks(1.0 + rank * 2.5, dist, torch, "cpu")
        q.put((rank, ms))
    finally:
        dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks_gloo():
    """The N>1 bench path (replicas, no data-path collective): the per-step time every
    rank prints is the maximum over ranks, computed with the same all-reduce on gloo."""
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_replica_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 3.5), (1, 3.5)]
