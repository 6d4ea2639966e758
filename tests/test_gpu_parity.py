"""Parity of the B200 engine with the oracle (CPU restatement of the reference operators)
on seeded tables: the same script runs through both and the STORE outputs must match
byte for byte (or as a multiset where the reference's row order is not defined)."""
import os

import pytest

import alenka_b200 as ab
from alenka_b200 import workloads as wl

from . import _oracle

pytestmark = pytest.mark.gpu


def _read(p):
    with open(p, "rb") as f:
        return f.read()


def _run_both(data_dir, script, out_name, plain=False, resident=True):
    _oracle.execute(data_dir, script.replace(out_name, "oracle_" + out_name))
    with ab.Session(data_dir, resident=resident, plain=plain) as s:
        s.execute(script)
        st = s.stats()
    return _read(os.path.join(data_dir, "oracle_" + out_name)), _read(os.path.join(data_dir, out_name)), st


@pytest.fixture(scope="module")
def flat_multi(tmp_path_factory):
    d = tmp_path_factory.mktemp("flat_multi")
    ab.gen_lineitem_flat(str(d), 300_000, 100_000, 11)
    return str(d)


@pytest.fixture(scope="module")
def flat_single(tmp_path_factory):
    d = tmp_path_factory.mktemp("flat_single")
    ab.gen_lineitem_flat(str(d), 250_000, 0, 12)
    return str(d)


@pytest.fixture(scope="module")
def flat_delta(tmp_path_factory):
    d = tmp_path_factory.mktemp("flat_delta")
    ab.gen_lineitem_flat(str(d), 200_000, 70_000, 13, delta=True)
    return str(d)


@pytest.fixture(scope="module")
def three_way(tmp_path_factory):
    d = tmp_path_factory.mktemp("three_way")
    wl.make_three_way(str(d), scale=0.01, seg_rows=200_000, seed=5)
    return str(d)


@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("plain", [True, False])
def test_flat_groupby_multi_segment(flat_multi, seed, plain):
    o, g, st = _run_both(flat_multi, wl.flat_script(seed), "q1.txt", plain=plain)
    assert o == g
    assert o.count(b"\n") == 5  # 3 x 2 groups
    assert st.rows_scanned > 0 and st.kernels > 0


@pytest.mark.parametrize("plain", [True, False])
def test_flat_groupby_single_segment_key_order(flat_single, plain):
    o, g, _ = _run_both(flat_single, wl.flat_script(4), "q1.txt", plain=plain)
    assert o == g


def test_flat_groupby_delta_segments(flat_delta):
    o, g, _ = _run_both(flat_delta, wl.flat_script(5), "q1.txt")
    assert o == g


@pytest.fixture(scope="module")
def three_way_delta(tmp_path_factory):
    d = tmp_path_factory.mktemp("three_way_delta")
    wl.make_three_way(str(d), scale=0.01, seg_rows=150_000, seed=8, delta=True)
    return str(d)


@pytest.mark.parametrize("seed", [1, 2])
def test_three_way_pipeline_delta_segments(three_way_delta, seed):
    # delta-encoded columns are expanded to int64 before the scan (64-bit evaluation path)
    o, g, _ = _run_both(three_way_delta, wl.three_way_script(seed), "q3.txt")
    assert o == g
    o, g = _run_both_or_error(three_way_delta, _three_way_with(*FUSED_PREDICATES["decimal"]), "fx.txt")
    assert o == g


@pytest.fixture(scope="module")
def three_way_skewed(tmp_path_factory):
    # the compressed config's shape: FOR-delta columns, lineitem's orderkeys Zipf(1.1)
    # over the orders (the heaviest order holds about 9% of the rows)
    d = tmp_path_factory.mktemp("three_way_skewed")
    wl.make_three_way(str(d), scale=0.02, seg_rows=300_000, seed=6, delta=True, zipf=1.1)
    return str(d)


@pytest.mark.parametrize("seed", [1, 2])
@pytest.mark.parametrize("plain", [True, False])
def test_three_way_skewed_delta(three_way_skewed, seed, plain):
    """Skewed join keys on FOR-delta segments, through the fused plan and the operator
    path, byte for byte against the oracle; every group, so the heavy keys' sums show."""
    o, g, st = _run_both(three_way_skewed, wl.three_way_script(seed, limit=0), "q3.txt", plain=plain)
    assert o == g
    assert o.count(b"\n") > 100
    o, g, st = _run_both(three_way_skewed, wl.three_way_script(seed), "q3.txt", plain=plain)
    assert o == g
    assert st.plan == (0 if plain else 1)  # LIMIT 10: the fused plan's device top-k


@pytest.mark.parametrize("seed", [1, 2])
@pytest.mark.parametrize("plain", [True, False])
def test_three_way_pipeline(three_way, seed, plain):
    o, g, _ = _run_both(three_way, wl.three_way_script(seed), "q3.txt", plain=plain)
    assert o == g
    assert o.count(b"\n") == 9


def test_three_way_pipeline_host_buffers(three_way):
    o, g, st = _run_both(three_way, wl.three_way_script(3), "q3.txt", resident=False)
    assert o == g
    assert st.h2d_bytes > 0


def test_three_way_full_group_output(three_way):
    # every group, in the reference's ORDER BY order with ties broken by group key order
    o, g, _ = _run_both(three_way, wl.three_way_script(4, limit=0), "q3.txt")
    assert o == g
    assert o.count(b"\n") > 100


SCRIPTS = {
    "and_or_decimal": (
        "LF := FILTER lineitem BY l_shipdate >= 19940101 AND l_quantity < 25 OR l_discount == 0.05;\n"
        "R := SELECT l_returnflag AS f, l_linestatus AS s, AVG(l_quantity) AS aq, MIN(l_extendedprice) AS mn, "
        "MAX(l_extendedprice) AS mx, COUNT(l_orderkey) AS c FROM LF GROUP BY l_returnflag, l_linestatus;\n"
        "STORE R INTO 'x.txt' USING ('|');\n"),
    "one_line": (
        "LF := FILTER lineitem BY l_shipdate < 19960101;\n"
        "S := SELECT SUM(l_quantity) AS q, COUNT(l_orderkey) AS c, MIN(l_extendedprice) AS mn, "
        "MAX(l_extendedprice) AS mx, AVG(l_quantity) AS a FROM LF;\n"
        "STORE S INTO 'x.txt' USING (',');\n"),
    "projection_order": (
        "LF := FILTER lineitem BY l_shipdate > 19980601;\n"
        "P := SELECT l_orderkey AS k, l_extendedprice*(1-l_discount) AS rev, l_shipdate AS d FROM LF;\n"
        "O := ORDER P BY rev DESC, d ASC;\n"
        "STORE O INTO 'x.txt' USING ('|') LIMIT 200;\n"),
    "strings": (
        "F := FILTER lineitem BY l_returnflag == \"R\" AND l_linestatus != \"O\";\n"
        "R := SELECT l_returnflag AS f, l_linestatus AS s, SUM(l_quantity) AS q, COUNT(l_orderkey) AS c "
        "FROM F GROUP BY l_returnflag, l_linestatus;\n"
        "STORE R INTO 'x.txt' USING ('|');\n"),
    "filter_arith": (
        "F := FILTER lineitem BY l_quantity*2 > 60 AND l_extendedprice - 1000.00 < 50000.00;\n"
        "R := SELECT l_linestatus AS s, SUM(l_extendedprice) AS p, COUNT(l_orderkey) AS c FROM F GROUP BY l_linestatus;\n"
        "STORE R INTO 'x.txt' USING ('|');\n"),
    "chained_filter_keys": (
        "F := FILTER lineitem BY l_shipdate < 19970101;\n"
        "G := FILTER F BY l_quantity > 10;\n"
        "R := SELECT l_orderkey AS k, SUM(l_quantity) AS q, COUNT(l_orderkey) AS c FROM G GROUP BY l_orderkey;\n"
        "O := ORDER R BY q DESC;\n"
        "STORE O INTO 'x.txt' USING ('|') LIMIT 100;\n"),
    "empty_filter": (
        "F := FILTER lineitem BY l_shipdate < 19000101;\n"
        "R := SELECT l_linestatus AS s, COUNT(l_orderkey) AS c FROM F GROUP BY l_linestatus;\n"
        "STORE R INTO 'x.txt' USING ('|');\n"),
}


@pytest.mark.parametrize("name", sorted(SCRIPTS))
@pytest.mark.parametrize("which", ["flat_multi", "flat_single"])
def test_scripts(name, which, request):
    d = request.getfixturevalue(which)
    o, g, _ = _run_both(d, SCRIPTS[name], "x.txt")
    assert o == g


def _three_way_with(lf, of, cf, limit=10):
    lim = f" LIMIT {limit}" if limit else ""
    return (f"OFI := FILTER orders BY {of};\n"
            f"CF := FILTER customer BY {cf};\n"
            f"LF := FILTER lineitem BY {lf};\n"
            "OLC := SELECT o_orderkey AS o_orderkey, o_orderdate AS o_orderdate, "
            "o_shippriority AS o_shippriority, l_extendedprice AS price, l_discount AS discount "
            "FROM LF JOIN OFI ON l_orderkey = o_orderkey JOIN CF ON o_custkey = c_custkey;\n"
            "F := SELECT o_orderkey AS o_orderkey1, o_orderdate AS orderdate1, o_shippriority AS priority, "
            "SUM(price*(1-discount)) AS sum_revenue, COUNT(o_orderkey) AS cnt "
            "FROM OLC GROUP BY o_orderkey, o_orderdate, o_shippriority;\n"
            "RES := ORDER F BY sum_revenue DESC, orderdate1 ASC;\n"
            f"STORE RES INTO 'fx.txt' USING ('|'){lim};\n")


# Fused-pipeline predicates: every comparison operator, constants inside, on and beyond
# the stored range (the scan rewrites conjuncts into unsigned tests on the stored FOR
# values), decimal-scaled constants, and predicates that are not conjunctions.
FUSED_PREDICATES = {
    "ge_le": ("l_shipdate >= 19950315", "o_orderdate <= 19950315", 'c_mktsegment == "BUILDING"'),
    "eq_ne": ("l_shipdate == 19950320", "o_orderdate != 19950301", 'c_mktsegment != "MACHINERY"'),
    "always": ("l_shipdate > 19000101", "o_orderdate < 20500101", 'c_mktsegment != "NOSUCHSEG"'),
    "never_fact": ("l_shipdate < 19000101", "o_orderdate < 19960101", 'c_mktsegment == "HOUSEHOLD"'),
    "never_dim": ("l_shipdate > 19940101", "o_orderdate > 20500101", 'c_mktsegment == "HOUSEHOLD"'),
    "decimal": ("l_discount > 0.05 AND l_extendedprice < 60000.00", "o_orderdate > 19960101 AND o_orderdate < 19970101",
                'c_mktsegment == "FURNITURE"'),
    "disjunction": ("l_shipdate < 19930301 OR l_shipdate > 19980101", "o_orderdate < 19930101 OR o_orderdate > 19971001",
                    'c_mktsegment == "AUTOMOBILE" OR c_mktsegment == "BUILDING"'),
    "three_conj": ("l_shipdate > 19950101 AND l_shipdate < 19950601 AND l_discount <= 0.03",
                   "o_orderdate >= 19941001", 'c_mktsegment == "BUILDING"'),
}


def _run_both_or_error(data_dir, script, out_name, plain=False):
    """Like _run_both, but a script the reference rejects must be rejected with the same
    message (an empty join leaves SELECT a column-less set, so ORDER BY cannot find its
    key: emit_select operators.cu:1847-1856, emit_order operators.cu:1641)."""
    try:
        _oracle.execute(data_dir, script.replace(out_name, "oracle_" + out_name))
    except RuntimeError as e:
        with ab.Session(data_dir, plain=plain) as s:
            with pytest.raises(ab.AlenkaError) as got:
                s.execute(script)
        assert str(e).split("oracle: ", 1)[1] in str(got.value)
        return None, None
    with ab.Session(data_dir, plain=plain) as s:
        s.execute(script)
    return _read(os.path.join(data_dir, "oracle_" + out_name)), _read(os.path.join(data_dir, out_name))


@pytest.mark.parametrize("plain", [False, True])
@pytest.mark.parametrize("name", sorted(FUSED_PREDICATES))
def test_fused_predicates(three_way, name, plain):
    o, g = _run_both_or_error(three_way, _three_way_with(*FUSED_PREDICATES[name]), "fx.txt", plain=plain)
    assert o == g


def test_fused_predicates_all_groups(three_way):
    o, g, _ = _run_both(three_way, _three_way_with(*FUSED_PREDICATES["decimal"], limit=0), "fx.txt")
    assert o == g


def test_fused_graph_capture_and_replay(three_way):
    """A resident session runs a fused query normally, captures it into a CUDA graph on its
    second run and replays the graph from the third; every run must store the oracle's
    rows. A second script interleaved with the first keeps its own graph."""
    scripts = [wl.three_way_script(7, out="rep_a.txt"), _three_way_with(*FUSED_PREDICATES["ge_le"])]
    outs = ["rep_a.txt", "fx.txt"]
    want = []
    for sc, o in zip(scripts, outs):
        _oracle.execute(three_way, sc.replace(o, "oracle_" + o))
        want.append(_read(os.path.join(three_way, "oracle_" + o)))
    with ab.Session(three_way, resident=True) as s:
        s.set_timing(True)
        for run in range(4):
            for sc, o, w in zip(scripts, outs, want):
                p = os.path.join(three_way, o)
                if os.path.exists(p):
                    os.remove(p)
                s.execute(sc)
                assert _read(p) == w, (o, run)
                st = s.stats()
                # plan 1: fused (runs 0 and 1, the second one captured), 2: replayed graph
                assert st.plan == (2 if run >= 2 else 1), (o, run, st.plan)
                assert st.kernels > 0 and st.rows_scanned > 0
                assert st.hot_kernel_launches == 1 and st.hot_kernel_ms > 0


def test_join_multiset(three_way):
    script = ("OFI := FILTER orders BY o_orderdate < 19950101;\n"
              "CF := FILTER customer BY c_mktsegment == \"BUILDING\";\n"
              "J := SELECT o_orderkey AS ok, o_orderdate AS od, c_custkey AS ck FROM OFI JOIN CF ON o_custkey = c_custkey;\n"
              "STORE J INTO 'j.txt' USING ('|');\n")
    o, g, _ = _run_both(three_way, script, "j.txt")
    assert sorted(o.split(b"\n")) == sorted(g.split(b"\n"))
    assert o.count(b"\n") > 100


def test_alenka_embedding_api(three_way, monkeypatch):
    """alenkaInit / alenkaExecute / alenkaClose with the current directory as data dir."""
    import ctypes
    monkeypatch.chdir(three_way)
    L = ab.lib()
    L.alenkaInit(None)
    try:
        script = wl.three_way_script(6, out="emb.txt")
        assert L.alenkaExecute(script.encode()) == 0
    finally:
        L.alenkaClose()
    _oracle.execute(three_way, wl.three_way_script(6, out="emb_oracle.txt"))
    assert _read(os.path.join(three_way, "emb.txt")) == _read(os.path.join(three_way, "emb_oracle.txt"))
    assert isinstance(ctypes, object)
