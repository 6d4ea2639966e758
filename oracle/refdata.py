"""Seeded synthetic tables in the reference's on-disk format, written with numpy alone.

Test infrastructure and CPU-baseline input only: the reference arm of the benchmark and
the golden-vector recipe use it to produce their tables without loading the product
library. It restates the product's seeded generators (splitmix64 streams, one stream
per column, the n-th draw a pure function of n) so that the same seed gives the same
bytes; a CPU test checks that file for file.

Formats written (FOR only, as the reference writes a column without the -delta flag):
  <table>.<col>.<seg>        segment image: u32 cnt | i64 lower | i64 upper | u32 comp |
                             payload | u32 cnt | u32 rows | u32 bits | i64 orig_lower |
                             u32 fit_count | i64 start_val   (pfor_compress,
                             compress.cu:413-527)
  <table>.<col>.header       u64 total | u32 segs | u32 max_recs | u32 max_cnt
                             (CudaSet::writeHeader, cm.cu:1251-1263)
  char columns               dictionary file <table>.<col> (fixed width, first-seen
                             order), <seg>.idx (FOR codes), <seg>.hash (u32 n + n x
                             MurmurHash64A(value, 100)/2)   (compress_char,
                             cm.cu:1765-1844)
  data.dictionary            catalog (save_col_data, cm.cu:4057-4080)
"""
import math
import os
import struct

import numpy as np

M64 = (1 << 64) - 1
GAMMA = 0x9E3779B97F4A7C15


def _mix(seed, stream):
    return (seed * GAMMA + stream * 0xD1B54A32D192ED03 + 1) & M64


def _draws(state, first, count):
    """splitmix64 outputs number first+1 .. first+count of a stream that starts at state."""
    n = np.arange(first + 1, first + count + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(state) + n * np.uint64(GAMMA)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def _uniform(state, first, count, lo, hi):
    """lo + draw % (hi - lo + 1), inclusive bounds, as int64."""
    span = np.uint64(hi - lo + 1)
    return (_draws(state, first, count) % span).astype(np.int64) + np.int64(lo)


def days_from_civil(y, m, d):
    y = y - (m <= 2)
    era = np.where(y >= 0, y, y - 399) // 400
    yoe = y - era * 400
    doy = (153 * (m + np.where(m > 2, -3, 9)) + 2) // 5 + d - 1
    doe = yoe * 365 + yoe // 4 - yoe // 100 + doy
    return era * 146097 + doe - 719468


def yyyymmdd(z):
    z = np.asarray(z, dtype=np.int64) + 719468
    era = np.where(z >= 0, z, z - 146096) // 146097
    doe = z - era * 146097
    yoe = (doe - doe // 1460 + doe // 36524 - doe // 146096) // 365
    y = yoe + era * 400
    doy = doe - (365 * yoe + yoe // 4 - yoe // 100)
    mp = (5 * doy + 2) // 153
    d = doy - (153 * mp + 2) // 5 + 1
    m = mp + np.where(mp < 10, 3, -9)
    y = y + (m <= 2)
    return y * 10000 + m * 100 + d


def date_add_days(v, days):
    y, m, d = v // 10000, (v // 100) % 100, v % 100
    return int(yyyymmdd(days_from_civil(np.int64(y), np.int64(m), np.int64(d)) + days))


def murmur64a(data: bytes, seed=100):
    """MurmurHash64A (MurmurHash2_64.cu:201-242), little-endian 8-byte blocks."""
    m, r = 0xC6A4A7935BD1E995, 47
    h = (seed ^ (len(data) * m)) & M64
    nb = len(data) // 8
    for i in range(nb):
        k = int.from_bytes(data[8 * i:8 * i + 8], "little")
        k = (k * m) & M64
        k ^= k >> r
        k = (k * m) & M64
        h ^= k
        h = (h * m) & M64
    tail = data[8 * nb:]
    if tail:
        for i in range(len(tail) - 1, -1, -1):
            h ^= tail[i] << (8 * i)
        h = (h * m) & M64
    h ^= h >> r
    h = (h * m) & M64
    h ^= h >> r
    return h


def _range_bits(lo, hi):
    span = ((hi - lo) & M64) + 1
    return int(math.ceil(math.log2(float(span))))


def _for_image(v):
    v = np.asarray(v, dtype=np.int64)
    n = len(v)
    lo = int(v.min()) if n else 0
    hi = int(v.max()) if n else 0
    bits = _range_bits(lo, hi)
    if bits not in (8, 16, 32, 64):
        bits = 8 if bits < 8 else 16 if bits < 16 else 32 if bits < 32 else 64
    dt = {8: np.uint8, 16: np.uint16, 32: np.uint32, 64: np.uint64}[bits]
    with np.errstate(over="ignore"):
        payload = (v.view(np.uint64) - np.uint64(lo & M64)).astype(dt).tobytes()
    cnt = len(payload)
    head = struct.pack("<IqqI", cnt, lo, hi, 0)
    tail = struct.pack("<IIIqIq", cnt, n, bits, lo, 64 // bits, 0)
    return head + payload + tail, cnt


class _Table:
    def __init__(self, d, name, cols):
        self.d, self.name, self.cols = d, name, cols  # cols: [(name, kind, decimals, width)]
        self.segs, self.total, self.max_recs = 0, 0, 0
        self.max_cnt = [0] * len(cols)
        self.dicts = [dict() for _ in cols]

    def segment(self, data):
        base = os.path.join(self.d, f"{self.name}.")
        rows = None
        for c, (cn, kind, _, width) in enumerate(self.cols):
            path = base + f"{cn}.{self.segs}"
            v = data[cn]
            if kind == 2:
                # v: uint8 array rows x width; dictionary codes by first appearance
                rows = len(v)
                uniq, first, inv = np.unique(v.view(f"S{width}").ravel() if width else v, return_index=True,
                                             return_inverse=True)
                hashes = {}
                codes_of_uniq = np.empty(len(uniq), dtype=np.int64)
                append = []
                for u in np.argsort(first, kind="stable"):
                    raw = bytes(v[first[u]].tobytes())
                    h = murmur64a(raw) // 2
                    hashes[u] = h
                    if h not in self.dicts[c]:
                        self.dicts[c][h] = len(self.dicts[c])
                        append.append(raw)
                    codes_of_uniq[u] = self.dicts[c][h]
                codes = codes_of_uniq[inv.ravel()]
                hv = np.array([hashes[u] for u in range(len(uniq))], dtype=np.uint64)[inv.ravel()]
                with open(base + cn, "ab" if self.segs else "wb") as f:
                    f.write(b"".join(append))
                with open(path + ".hash", "wb") as f:
                    f.write(struct.pack("<I", rows) + hv.astype("<u8").tobytes())
                v = codes
                path += ".idx"
            rows = len(v)
            img, cnt = _for_image(v)
            with open(path, "wb") as f:
                f.write(img)
            self.max_cnt[c] = max(self.max_cnt[c], cnt)
        self.segs += 1
        self.total += rows
        self.max_recs = max(self.max_recs, rows)

    def finish(self, catalog):
        for c, (cn, kind, dec, width) in enumerate(self.cols):
            with open(os.path.join(self.d, f"{self.name}.{cn}.header"), "wb") as f:
                f.write(struct.pack("<QIII", self.total, self.segs, self.max_recs, self.max_cnt[c]))
            catalog.setdefault(self.name, {})[cn] = (2 if kind == 2 else 0,
                                                     dec if kind == 1 else (width if kind == 2 else 0))


def _load_catalog(path):
    cat = {}
    if not os.path.exists(path):
        return cat
    b = open(path, "rb").read()
    off = 0

    def u64():
        nonlocal off
        v = struct.unpack_from("<Q", b, off)[0]
        off += 8
        return v
    for _ in range(u64()):
        ln = u64()
        t = b[off:off + ln].decode()
        off += ln
        for _ in range(u64()):
            cl = u64()
            c = b[off:off + cl].decode()
            off += cl
            cat.setdefault(t, {})[c] = struct.unpack_from("<II", b, off)
            off += 8
    return cat


def _save_catalog(path, cat):
    out = [struct.pack("<Q", len(cat))]
    for t in sorted(cat):
        tb = t.encode()
        out.append(struct.pack("<Q", len(tb)) + tb + struct.pack("<Q", len(cat[t])))
        for c in sorted(cat[t]):
            cb = c.encode()
            out.append(struct.pack("<Q", len(cb)) + cb + struct.pack("<II", *cat[t][c]))
    with open(path, "wb") as f:
        f.write(b"".join(out))


def _write(d, name, cols, columns, rows, seg_rows, cat):
    """columns: name -> array over all rows, or a function (begin, end) -> that slice
    (so that large tables are produced one segment at a time)."""
    t = _Table(d, name, cols)
    seg_rows = seg_rows or rows
    for b in range(0, rows, seg_rows):
        e = min(rows, b + seg_rows)
        t.segment({k: (v(b, e) if callable(v) else v[b:e]) for k, v in columns.items()})
    t.finish(cat)


def _order_counts(state, rows):
    """Prefix ends of the per-order row counts (1-7, one draw per order) until they cover
    rows: cum[k] = rows of orders 0..k."""
    k = rows // 4 + 64
    while True:
        cum = np.cumsum(_uniform(state, 0, k, 1, 7))
        if int(cum[-1]) >= rows:
            return cum
        k *= 2


SEGMENTS = [b"AUTOMOBILE", b"BUILDING", b"FURNITURE", b"HOUSEHOLD", b"MACHINERY"]


def three_way(d, customers, orders, lineitems, seg_rows, seed):
    """customer (custkey 1..C, mktsegment of 5 values), orders (orderkey 4*i, custkey
    uniform, orderdate uniform over 7 years from 1992-01-01, shippriority 0), lineitem
    (orderkey with 1-7 rows per order in order, wrapping to the first order when the
    orders run out, shipdate = orderdate + U[1,121] days, extendedprice cents
    U[90000,10500000], discount U[0,10] hundredths)."""
    cat = _load_catalog(os.path.join(d, "data.dictionary"))
    seg = _uniform(_mix(seed, 11), 0, customers, 0, 4)
    names = np.zeros((customers, 10), dtype=np.uint8)
    table = np.frombuffer(b"".join(s.ljust(10, b"\0") for s in SEGMENTS), dtype=np.uint8).reshape(5, 10)
    names[:] = table[seg]
    _write(d, "customer", [("c_custkey", 0, 0, 0), ("c_mktsegment", 2, 0, 10)],
           {"c_custkey": np.arange(1, customers + 1, dtype=np.int64), "c_mktsegment": names},
           customers, seg_rows, cat)
    del names, seg
    d0 = int(days_from_civil(np.int64(1992), np.int64(1), np.int64(1)))
    odays = _uniform(_mix(seed, 22), 0, orders, d0, d0 + 7 * 365 - 1)
    _write(d, "orders", [("o_orderkey", 0, 0, 0), ("o_custkey", 0, 0, 0), ("o_orderdate", 0, 0, 0),
                         ("o_shippriority", 0, 0, 0)],
           {"o_orderkey": lambda b, e: 4 * np.arange(b + 1, e + 1, dtype=np.int64),
            "o_custkey": lambda b, e: _uniform(_mix(seed, 21), b, e - b, 1, customers),
            "o_orderdate": lambda b, e: yyyymmdd(odays[b:e]),
            "o_shippriority": lambda b, e: np.zeros(e - b, dtype=np.int64)},
           orders, seg_rows, cat)
    cum = _order_counts(_mix(seed, 31), lineitems)

    def order_of(b, e):  # the order a lineitem row belongs to; the order list wraps around
        return np.searchsorted(cum, np.arange(b, e, dtype=np.int64), side="right") % orders
    _write(d, "lineitem", [("l_orderkey", 0, 0, 0), ("l_shipdate", 0, 0, 0), ("l_extendedprice", 1, 2, 0),
                           ("l_discount", 1, 2, 0)],
           {"l_orderkey": lambda b, e: 4 * (order_of(b, e) + 1),
            "l_shipdate": lambda b, e: yyyymmdd(odays[order_of(b, e)] + _uniform(_mix(seed, 32), b, e - b, 1, 121)),
            "l_extendedprice": lambda b, e: _uniform(_mix(seed, 33), b, e - b, 90000, 10500000),
            "l_discount": lambda b, e: _uniform(_mix(seed, 34), b, e - b, 0, 10)},
           lineitems, seg_rows, cat)
    _save_catalog(os.path.join(d, "data.dictionary"), cat)


def lineitem_flat(d, rows, seg_rows, seed):
    """Single-table lineitem: orderkey (1-7 rows per key), quantity U[1,50], extendedprice
    cents U[90000,10500000], discount U[0,10], shipdate uniform over 1992-01-02..1998-12-01,
    returnflag in {A,N,R}, linestatus in {F,O}."""
    cat = _load_catalog(os.path.join(d, "data.dictionary"))
    cum = _order_counts(_mix(seed, 1), rows)
    keys = np.searchsorted(cum, np.arange(rows, dtype=np.int64), side="right") + 1
    d0 = int(days_from_civil(np.int64(1992), np.int64(1), np.int64(2)))
    d1 = int(days_from_civil(np.int64(1998), np.int64(12), np.int64(1)))
    flags = np.frombuffer(b"ANR", dtype=np.uint8)[_uniform(_mix(seed, 6), 0, rows, 0, 2)].reshape(rows, 1)
    stat = np.frombuffer(b"FO", dtype=np.uint8)[_uniform(_mix(seed, 7), 0, rows, 0, 1)].reshape(rows, 1)
    _write(d, "lineitem", [("l_orderkey", 0, 0, 0), ("l_quantity", 0, 0, 0), ("l_extendedprice", 1, 2, 0),
                           ("l_discount", 1, 2, 0), ("l_shipdate", 0, 0, 0), ("l_returnflag", 2, 0, 1),
                           ("l_linestatus", 2, 0, 1)],
           {"l_orderkey": keys, "l_quantity": _uniform(_mix(seed, 2), 0, rows, 1, 50),
            "l_extendedprice": _uniform(_mix(seed, 3), 0, rows, 90000, 10500000),
            "l_discount": _uniform(_mix(seed, 4), 0, rows, 0, 10),
            "l_shipdate": yyyymmdd(_uniform(_mix(seed, 5), 0, rows, d0, d1)),
            "l_returnflag": np.ascontiguousarray(flags), "l_linestatus": np.ascontiguousarray(stat)},
           rows, seg_rows, cat)
    _save_catalog(os.path.join(d, "data.dictionary"), cat)
