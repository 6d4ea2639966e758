"""Parity pinned to the reference itself: every case in tests/golden/ref_ops/manifest.json
holds what the reference's own operators (built for the CPU from its sources, Thrust's
OpenMP device system, tests/golden/make_ref_ops.py) stored for a script over seeded
tables. The oracle (CPU) and the engine (GPU; fused and plain plans) must store the same
bytes, the same multiset of rows where the reference defines no row order, or stop with
the same fatal error. Inputs are checked against the digest the reference saw."""
import hashlib
import json
import os
import shutil

import pytest

from oracle import refdata
from . import _oracle
from . import ref_cases

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "ref_ops")
MANIFEST = json.load(open(os.path.join(GOLD, "manifest.json")))
CASES = {c["name"]: c for c in MANIFEST["cases"]}
CPU_ROWS = 10_000_000  # datasets the CPU suite builds and runs through the oracle


def _digest_dir(d):
    h = hashlib.sha256()
    for f in sorted(os.listdir(d)):
        p = os.path.join(d, f)
        if not os.path.isfile(p) or f.endswith((".sql", ".txt")):
            continue
        h.update(f.encode() + b"\0")
        with open(p, "rb") as fh:
            while True:
                b = fh.read(1 << 24)
                if not b:
                    break
                h.update(b)
    return h.hexdigest()


class _ProductGen:
    """The product's generators behind refdata's interface (same bytes, faster)."""

    @staticmethod
    def lineitem_flat(d, rows, seg_rows, seed):
        import alenka_b200 as ab
        ab.gen_lineitem_flat(d, rows, seg_rows, seed)

    @staticmethod
    def three_way(d, customers, orders, rows, seg_rows, seed):
        import alenka_b200 as ab
        ab.gen_three_way(d, customers, orders, rows, seg_rows, seed)


_made = {}


def _dataset(name, tmp_path_factory, gen):
    if name not in _made:
        d = str(tmp_path_factory.mktemp("ref_" + name))
        ref_cases.make_dataset(d, MANIFEST["datasets"][name], gen)
        _made[name] = d
    d = _made[name]
    for c in MANIFEST["cases"]:
        if c["dataset"] == name:
            assert _digest_dir(d) == c["data_sha256"], f"{name}: tables differ from those the reference read"
            break
    return d


def _want(case):
    if "file" in case:
        return open(os.path.join(GOLD, case["file"]), "rb").read()
    return None


def _check(case, got):
    want = _want(case)
    if case["mode"] == "multiset":
        lines = sorted(got.split(b"\n"))
        if want is not None:
            assert lines == sorted(want.split(b"\n")), case["name"]
        else:
            assert got.count(b"\n") == case["lines"], case["name"]
            assert hashlib.sha256(b"\n".join(lines)).hexdigest() == case["sorted_sha256"], case["name"]
    elif want is not None:
        assert got == want, case["name"]
    else:
        assert got.count(b"\n") == case["lines"], case["name"]
        assert hashlib.sha256(got).hexdigest() == case["sha256"], case["name"]


def _rows(case):
    return MANIFEST["datasets"][case["dataset"]]["rows"]


CPU_CASES = sorted(n for n, c in CASES.items() if _rows(c) < CPU_ROWS)


def test_refdata_writes_the_product_generators_bytes(tmp_path):
    import filecmp
    import alenka_b200 as ab
    for kind, args in [("three", (3000, 30000, 120123, 50000, 5)), ("three", (1500, 15000, 70000, 0, 9)),
                       ("flat", (123457, 40000, 11))]:
        a, b = tmp_path / f"p{kind}{args[-1]}", tmp_path / f"r{kind}{args[-1]}"
        a.mkdir()
        b.mkdir()
        if kind == "three":
            ab.gen_three_way(str(a), *args)
            refdata.three_way(str(b), *args)
        else:
            ab.gen_lineitem_flat(str(a), *args)
            refdata.lineitem_flat(str(b), *args)
        fa, fb = sorted(os.listdir(a)), sorted(os.listdir(b))
        assert fa == fb
        for f in fa:
            assert filecmp.cmp(a / f, b / f, shallow=False), f


@pytest.mark.parametrize("name", CPU_CASES)
def test_oracle_matches_reference(name, tmp_path_factory):
    case = CASES[name]
    d = _dataset(case["dataset"], tmp_path_factory, refdata)
    out = "oracle_" + case["out"]
    script = case["script"].replace(f"'{case['out']}'", f"'{out}'")
    if "error" in case:
        with pytest.raises(RuntimeError) as e:
            _oracle.execute(d, script)
        assert str(e.value) == "oracle: " + case["error"]
        return
    _oracle.execute(d, script)
    _check(case, open(os.path.join(d, out), "rb").read())


REF_BIN = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "alenka_ref")


@pytest.mark.skipif(not os.path.exists(REF_BIN), reason="reference build absent (oracle/build_ref.sh)")
@pytest.mark.parametrize("name", ["flat_multi_q1_s1", "three_way_q3_s1", "three_way_join_alias_scale"])
def test_reference_build_reproduces_its_golden_output(name, tmp_path):
    import subprocess
    case = CASES[name]
    ref_cases.make_dataset(str(tmp_path), MANIFEST["datasets"][case["dataset"]], refdata)
    (tmp_path / "g.sql").write_text(case["script"])
    subprocess.run([REF_BIN, "g.sql"], cwd=tmp_path, check=True, capture_output=True, timeout=600)
    _check(case, (tmp_path / case["out"]).read_bytes())


def _engine(case, d, plain):
    import alenka_b200 as ab
    out = ("plain_" if plain else "gpu_") + case["out"]
    script = case["script"].replace(f"'{case['out']}'", f"'{out}'")
    with ab.Session(d, plain=plain) as s:
        if "error" in case:
            with pytest.raises(ab.AlenkaError) as e:
                s.execute(script)
            assert case["error"] in str(e.value)
            return
        s.execute(script)
        st = s.stats()
    _check(case, open(os.path.join(d, out), "rb").read())
    if "segments_skipped" in case:  # segments whose zone-map verdict is N are never read
        assert st.segments_skipped == case["segments_skipped"], (case["name"], st.segments_skipped)


@pytest.mark.gpu
@pytest.mark.parametrize("plain", [False, True])
@pytest.mark.parametrize("name", sorted(CASES))
def test_engine_matches_reference(name, plain, tmp_path_factory):
    case = CASES[name]
    d = _dataset(case["dataset"], tmp_path_factory, _ProductGen)
    _engine(case, d, plain)


def teardown_module(module):
    for d in _made.values():
        shutil.rmtree(d, ignore_errors=True)
    _made.clear()
