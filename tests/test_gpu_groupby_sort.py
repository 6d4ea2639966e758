"""Sort-based group-by (the reference's own form) against the hash group-by and the oracle.

alk_groupby_sort and alk_groupby_hash on the same inputs must give the same groups, the
same exact int64 aggregates and the same first row per group (compared as maps: the hash
form's group order is unspecified); the in-order check must skip the sort exactly when
the key tuples are non-decreasing. Through the engine, a high-cardinality GROUP BY runs
in either form and matches the oracle byte for byte."""
import ctypes as c
import os

import numpy as np
import pytest

import alenka_b200 as ab
from alenka_b200 import workloads as wl

from .test_gpu_parity import _run_both_or_error

pytestmark = pytest.mark.gpu

SUM, COUNT, MIN, MAX = 0, 1, 2, 3


def _lib():
    L = ab.lib()
    vp, u32, u64 = c.c_void_p, c.c_uint32, c.c_uint64
    L.alk_groupby_sort.argtypes = [c.POINTER(vp), u32, c.POINTER(vp), c.POINTER(c.c_uint8), u32, u64, c.POINTER(vp),
                                   c.POINTER(vp), vp, c.POINTER(u64), c.POINTER(c.c_int), vp]
    return L


def _run(form, keys, vals, kinds):
    import torch
    L = _lib()
    n = len(keys[0])
    dk = [torch.from_numpy(np.ascontiguousarray(k)).cuda() for k in keys]
    dv = [torch.from_numpy(np.ascontiguousarray(v)).cuda() for v in vals]
    ok = [torch.zeros(n, dtype=torch.int64, device="cuda") for _ in keys]
    ov = [torch.zeros(n, dtype=torch.int64, device="cuda") for _ in vals]
    first = torch.zeros(n, dtype=torch.int32, device="cuda")
    P = lambda ts: (c.c_void_p * len(ts))(*[t.data_ptr() for t in ts])
    g = c.c_uint64()
    ag = (c.c_uint8 * len(kinds))(*kinds)
    in_order = c.c_int(-1)
    if form == "sort":
        rc = L.alk_groupby_sort(P(dk), len(keys), P(dv), ag, len(vals), n, P(ok), P(ov), c.c_void_p(first.data_ptr()),
                                c.byref(g), c.byref(in_order), None)
    else:
        rc = L.alk_groupby_hash(P(dk), len(keys), P(dv), ag, len(vals), n, P(ok), P(ov),
                                c.c_void_p(first.data_ptr()), c.byref(g), None)
    assert rc == 0
    torch.cuda.synchronize()
    G = g.value
    K = [k[:G].cpu().numpy() for k in ok]
    V = [v[:G].cpu().numpy() for v in ov]
    F = first[:G].cpu().numpy()
    out = {tuple(int(k[i]) for k in K): (tuple(int(v[i]) for v in V), int(F[i])) for i in range(G)}
    assert len(out) == G
    return out, K, in_order.value


@pytest.mark.parametrize("order", ["random", "sorted"])
@pytest.mark.parametrize("nkeys", [1, 2])
def test_sort_equals_hash(order, nkeys):
    rng = np.random.default_rng(nkeys * 7 + (order == "sorted"))
    n = 1_000_003
    keys = [rng.integers(-50_000, 50_000, n).astype(np.int64)]
    if nkeys == 2:
        keys.append(rng.integers(-3, 4, n).astype(np.int64))
    if order == "sorted":
        idx = np.lexsort(tuple(reversed(keys)))
        keys = [k[idx] for k in keys]
    vals = [rng.integers(-2**40, 2**40, n).astype(np.int64) for _ in range(4)]
    kinds = [SUM, MIN, MAX, COUNT]
    hs, _, _ = _run("hash", keys, vals, kinds)
    ss, K, in_order = _run("sort", keys, vals, kinds)
    assert in_order == (1 if order == "sorted" else 0)
    assert hs == ss
    # the sort form's groups come out in key order
    t = list(zip(*[k.tolist() for k in K]))
    assert t == sorted(t)


def test_sort_edge_cases():
    # one row; all rows one key; keys at the int64 extremes
    for keys in ([np.array([5], np.int64)], [np.full(70_000, 9, np.int64)],
                 [np.array([2**63 - 1, -2**63, 0, -2**63, 2**63 - 1], np.int64)]):
        vals = [np.arange(len(keys[0]), dtype=np.int64)]
        hs, _, _ = _run("hash", keys, vals, [SUM])
        ss, _, _ = _run("sort", keys, vals, [SUM])
        assert hs == ss


@pytest.fixture(scope="module")
def flat(tmp_path_factory):
    d = tmp_path_factory.mktemp("gbsort")
    ab.gen_lineitem_flat(str(d), 300_000, 100_000, 41)
    return str(d)


HIGH = ("LF := FILTER lineitem BY l_shipdate < 19960101;\n"
        "R := SELECT l_orderkey AS k, SUM(l_quantity) AS q, SUM(l_extendedprice*(1-l_discount)) AS rev, "
        "MIN(l_discount) AS mn, COUNT(l_orderkey) AS c FROM LF GROUP BY l_orderkey;\n"
        "STORE R INTO 'hs.txt' USING ('|');\n")


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_engine_high_cardinality_groupby(flat, mode):
    from . import _oracle
    _oracle.execute(flat, HIGH.replace("hs.txt", "oracle_hs.txt"))
    want = open(os.path.join(flat, "oracle_hs.txt"), "rb").read()
    with ab.Session(flat) as s:
        s.set_groupby(mode)
        s.execute(HIGH)
        st = s.stats()
        assert st.sort_groupbys == (1 if mode == 2 else 0)
        assert st.hash_groupbys == (0 if mode == 2 else 1)  # the filter and the hashing in one pass
    assert open(os.path.join(flat, "hs.txt"), "rb").read() == want


FUSED = {
    # one key column whose range is too wide to index directly: the one-CAS hash table
    "wide_key": "LF := FILTER lineitem BY l_shipdate >= 19950101;\n"
                "R := SELECT l_extendedprice AS p, SUM(l_quantity) AS q, MIN(l_discount) AS mn, "
                "COUNT(l_orderkey) AS c FROM LF GROUP BY l_extendedprice;\n"
                "STORE R INTO 'fz.txt' USING ('|');\n",
    # two unsorted key columns (the multi-column hash table), MAX and an expression input
    "two_keys": "LF := FILTER lineitem BY l_shipdate < 19960101 AND l_quantity > 10;\n"
                "R := SELECT l_extendedprice AS p, l_discount AS d, SUM(l_quantity) AS q, MAX(l_shipdate) AS mx, "
                "COUNT(l_orderkey) AS c FROM LF GROUP BY l_extendedprice, l_discount;\n"
                "STORE R INTO 'fz.txt' USING ('|');\n",
    # a predicate that is not a conjunction runs per row
    "or_pred": "LF := FILTER lineitem BY l_shipdate < 19930101 OR l_quantity == 7;\n"
               "R := SELECT l_orderkey AS k, SUM(l_extendedprice*(1-l_discount)) AS rev, MIN(l_quantity) AS mn, "
               "COUNT(l_orderkey) AS c FROM LF GROUP BY l_orderkey;\n"
               "STORE R INTO 'fz.txt' USING ('|');\n",
    # the base table itself, no filter; char-coded keys
    "base_char": "R := SELECT l_returnflag AS f, l_linestatus AS s, l_quantity AS q, SUM(l_extendedprice) AS p, "
                 "COUNT(l_orderkey) AS c FROM lineitem GROUP BY l_returnflag, l_linestatus, l_quantity;\n"
                 "STORE R INTO 'fz.txt' USING ('|');\n",
    # zone maps skip the first segment: the reference then reverses the select list
    "first_empty": "LF := FILTER lineitem BY l_orderkey > 30000;\n"
                   "R := SELECT l_orderkey AS k, SUM(l_quantity) AS q, COUNT(l_orderkey) AS c FROM LF "
                   "GROUP BY l_orderkey;\nSTORE R INTO 'fz.txt' USING ('|');\n",
    # nothing survives
    "empty": "LF := FILTER lineitem BY l_quantity > 60;\n"
             "R := SELECT l_orderkey AS k, SUM(l_quantity) AS q, COUNT(l_orderkey) AS c FROM LF "
             "GROUP BY l_orderkey;\nSTORE R INTO 'fz.txt' USING ('|');\n",
}


@pytest.mark.parametrize("name", sorted(FUSED))
def test_fused_hash_groupby_matches_oracle(flat, name):
    """The fused filter + hash GROUP BY (alk_pipeline_groupby) through the engine, byte
    for byte against the oracle, in its three forms: the key space indexing the
    accumulators (l_orderkey; the char-coded keys), a one-column hash table (a key range
    wider than 16 slots per row) and a multi-column one. Also predicates that are and are
    not conjunctions, no filter, a skipped first segment, and an empty result."""
    from . import _oracle
    script = FUSED[name]
    _oracle.execute(flat, script.replace("fz.txt", "oracle_fz.txt"))
    with ab.Session(flat) as s:
        s.set_groupby(1)
        s.execute(script)
        # with every segment skipped the key range is empty, and the dense form takes it
        assert s.stats().hash_groupbys == (0 if name == "empty" else 1)
    assert open(os.path.join(flat, "fz.txt"), "rb").read() == open(os.path.join(flat, "oracle_fz.txt"), "rb").read()


def test_engine_sort_form_small_keys(flat):
    # the config-1 group-by through the operator path in its sort-based form
    script = wl.flat_script(9, out="ss.txt")
    from . import _oracle
    _oracle.execute(flat, script.replace("ss.txt", "oracle_ss.txt"))
    with ab.Session(flat, plain=True) as s:
        s.set_groupby(2)
        s.execute(script)
        assert s.stats().sort_groupbys == 1
    assert open(os.path.join(flat, "ss.txt"), "rb").read() == open(os.path.join(flat, "oracle_ss.txt"), "rb").read()
