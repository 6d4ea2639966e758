"""Star join with bitmap join indexes, pinned to the reference: tests/golden/star holds what
the reference's own CREATE INDEX and star join wrote for tests/star_cases.py (index file
digests and stored results, tests/golden/make_star.py). The oracle (CPU) and the engine
(GPU) must write the same index files and store the same bytes, or stop with the same
error; at a larger size the engine must agree with the oracle byte for byte."""
import hashlib
import json
import os
import shutil

import pytest

from oracle import refdata
from . import _oracle
from . import star_cases
from .test_ref_golden import _digest_dir, _ProductGen

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "star")
MANIFEST = json.load(open(os.path.join(GOLD, "manifest.json")))
CASES = {c["name"]: c for c in MANIFEST["cases"]}

_made = {}


def _dataset(name, tmp_path_factory, gen, tag):
    """The dataset with its indexes built by `tag` ("oracle" or "engine")."""
    key = (name, tag)
    if key not in _made:
        d = str(tmp_path_factory.mktemp(f"star_{name}_{tag}"))
        star_cases.make_dataset(d, MANIFEST["datasets"][name], gen)
        assert _digest_dir(d) == MANIFEST["indexes"][name]["data_sha256"], "tables differ from the reference's"
        if tag == "oracle":
            _oracle.execute(d, MANIFEST["setup"][name])
        else:
            import alenka_b200 as ab
            with ab.Session(d) as s:
                s.execute(MANIFEST["setup"][name])
        _made[key] = d
    return _made[key]


def _index_digests(d, name):
    return {f: hashlib.sha256(open(os.path.join(d, f), "rb").read()).hexdigest()
            for f in MANIFEST["indexes"][name]["files"]}


def _check(case, got):
    if "file" in case:
        assert got == open(os.path.join(GOLD, case["file"]), "rb").read(), case["name"]
    else:
        assert got.count(b"\n") == case["lines"], case["name"]
        assert hashlib.sha256(got).hexdigest() == case["sha256"], case["name"]


def _renamed(case, prefix):
    out = prefix + case["out"]
    return out, case["script"].replace(f"'{case['out']}'", f"'{out}'")


# ---------------------------------------------------------------- CPU: the oracle
@pytest.mark.parametrize("name", sorted(MANIFEST["indexes"]))
def test_oracle_writes_the_reference_index_files(name, tmp_path_factory):
    d = _dataset(name, tmp_path_factory, refdata, "oracle")
    assert _index_digests(d, name) == MANIFEST["indexes"][name]["files"]


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_star_join_matches_reference(name, tmp_path_factory):
    case = CASES[name]
    d = _dataset(case["dataset"], tmp_path_factory, refdata, "oracle")
    out, script = _renamed(case, "oracle_")
    if "error" in case:
        with pytest.raises(RuntimeError) as e:
            _oracle.execute(d, script)
        assert str(e.value) == "oracle: " + case["error"]
        return
    _oracle.execute(d, script)
    _check(case, open(os.path.join(d, out), "rb").read())


def test_oracle_refuses_a_statement_after_create_index(tmp_path_factory):
    # the reference's CREATE INDEX leaves its names queued for the next statement
    d = _dataset("star_b", tmp_path_factory, refdata, "oracle")
    with pytest.raises(RuntimeError, match="after CREATE INDEX"):
        _oracle.execute(d, MANIFEST["setup"]["star_b"] + CASES["b_segment"]["script"])


FRONTEND_DUMP = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "frontend_dump")


@pytest.mark.skipif(not os.path.exists(FRONTEND_DUMP), reason="reference front end absent (oracle/build_ref.sh)")
def test_reference_grammar_queues_the_star_scripts_as_the_engine_parser(tmp_path):
    from .test_frontend import _engine_dump, _reference_dump
    for script in list(MANIFEST["setup"].values()) + [c["script"] for c in MANIFEST["cases"]]:
        rc, want = _engine_dump(script)
        assert rc == 0, want
        rrc, got = _reference_dump(script, tmp_path)
        assert rrc == 0
        assert got == want, script


# ---------------------------------------------------------------- GPU: the engine
@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(MANIFEST["indexes"]))
def test_engine_writes_the_reference_index_files(name, tmp_path_factory):
    d = _dataset(name, tmp_path_factory, _ProductGen, "engine")
    assert _index_digests(d, name) == MANIFEST["indexes"][name]["files"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_engine_star_join_matches_reference(name, tmp_path_factory):
    import alenka_b200 as ab
    case = CASES[name]
    d = _dataset(case["dataset"], tmp_path_factory, _ProductGen, "engine")
    out, script = _renamed(case, "gpu_")
    with ab.Session(d) as s:
        if "error" in case:
            with pytest.raises(ab.AlenkaError) as e:
                s.execute(script)
            assert case["error"] in str(e.value)
            return
        s.execute(script)
    _check(case, open(os.path.join(d, out), "rb").read())


@pytest.mark.gpu
def test_engine_refuses_a_statement_after_create_index(tmp_path_factory):
    import alenka_b200 as ab
    d = _dataset("star_b", tmp_path_factory, _ProductGen, "engine")
    with ab.Session(d) as s:
        with pytest.raises(ab.AlenkaError, match="after CREATE INDEX"):
            s.execute(MANIFEST["setup"]["star_b"] + CASES["b_segment"]["script"])


@pytest.mark.gpu
def test_engine_star_join_matches_oracle_at_6m_rows(tmp_path):
    """lineitem 6M rows in three segments, orders 1.5M and customer 150k in one: the engine's
    index files and star join results equal the oracle's byte for byte."""
    import alenka_b200 as ab
    a, b = tmp_path / "engine", tmp_path / "oracle"
    a.mkdir()
    ab.gen_three_way(str(a), 150_000, 1_500_000, 6_000_000, 2_000_000, 11)
    shutil.copytree(a, b)
    setup = ("CREATE INDEX lo ON lineitem(orders.o_orderdate) FROM lineitem, orders "
             "WHERE lineitem.l_orderkey = orders.o_orderkey;\n"
             "CREATE INDEX oc ON orders(customer.c_mktsegment) FROM orders, customer "
             "WHERE orders.o_custkey = customer.c_custkey;\n")
    q1 = ("LF := FILTER lineitem BY l_shipdate < 19940101;\n"
          "OF := FILTER orders BY o_orderdate == 19930704 OR o_orderdate == 19931111 OR o_orderdate > 19920101;\n"
          "J := SELECT l_orderkey AS l_orderkey, l_extendedprice AS l_extendedprice, o_orderdate AS o_orderdate "
          "FROM LF JOIN OF ON l_orderkey = o_orderkey;\n"
          "STORE J INTO 'q1.txt' USING ('|');\n")
    q2 = ('CF := FILTER customer BY c_mktsegment == "AUTOMOBILE";\n'
          "J := SELECT o_orderkey AS o_orderkey, o_custkey AS o_custkey, c_mktsegment AS c_mktsegment "
          "FROM orders JOIN CF ON o_custkey = c_custkey;\n"
          "G := SELECT c_mktsegment AS seg, COUNT(o_orderkey) AS cnt, SUM(o_custkey) AS s FROM J GROUP BY c_mktsegment;\n"
          "STORE G INTO 'q2.txt' USING ('|');\n")
    with ab.Session(str(a)) as s:
        s.execute(setup)
        s.execute(q1)
        s.execute(q2)
    _oracle.execute(str(b), setup)
    _oracle.execute(str(b), q1)
    _oracle.execute(str(b), q2)
    files = [f for f in os.listdir(b) if f.startswith(("lineitem.orders.", "orders.customer."))]
    assert len(files) == 4
    for f in sorted(files) + ["q1.txt", "q2.txt"]:
        assert (a / f).read_bytes() == (b / f).read_bytes(), f
    assert (a / "q1.txt").read_bytes().count(b"\n") > 1000


def teardown_module(module):
    for d in _made.values():
        shutil.rmtree(d, ignore_errors=True)
    _made.clear()
