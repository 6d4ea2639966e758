"""The reference's own script front end on this engine, through the operator-level
boundary (include/alenka_b200_operators.h): the reference's generated parser (bison.cu,
lex.yy.c), its CLI (main.cu) and error callbacks (callbacks.c), compiled from its sources
and linked against libalenka_b200.so in place of its operators (oracle/ref.mk, target
frontend: oracle/_ref/alenka_frontend and oracle/_ref/frontend_dump).

CPU: the header's declarations are all exported; the reference grammar's actions, seen
through the boundary, queue exactly what the engine's own parser queues for the same
script (golden scripts plus a corpus of the grammar's other statement forms), and both
reject what the grammar rejects. GPU: the reference CLI run on golden tables stores the
reference's own output, byte for byte, and stops with its fatal error where it does."""
import ctypes
import os
import re
import subprocess

import pytest

import alenka_b200 as ab

from . import ref_cases
from . import test_ref_golden as gold

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
DUMP = os.path.join(REF, "frontend_dump")
CLI = os.path.join(REF, "alenka_frontend")
HDR = os.path.join(ROOT, "include", "alenka_b200_operators.h")

CORPUS = [
    # LOAD, FILTER with OR / decimal / string, every aggregate, ORDER, STORE forms, DISPLAY
    "A := LOAD 'file.tbl' USING ('|') AS (a{1}:int, b{2}:varchar(10), c{3}:decimal(10,2));\n"
    "B := FILTER A BY a > 5 AND b == \"xyz\" OR c <= 1.50;\n"
    "C := SELECT a AS a, SUM(c) AS s, AVG(c) AS av, MIN(a) AS mn, MAX(a) AS mx, COUNT(a) AS cnt FROM B GROUP BY a;\n"
    "D := ORDER C BY s DESC, a ASC;\n"
    "STORE D INTO 'out.txt' USING ('|') LIMIT 5;\n"
    "STORE D INTO 'dbin' BINARY;\n"
    "STORE D INTO 'dbin' APPEND BINARY;\n"
    "DISPLAY D USING ('|') LIMIT 3;\n",
    # multi-column, semi / anti and chained joins, date parts, CAST, LIKE, != and negatives
    "J := SELECT a AS a, x AS x FROM B JOIN E ON a = x AND b = y;\n"
    "K := SELECT a AS a FROM B LEFT SEMI JOIN E ON a = x;\n"
    "L := SELECT a AS a FROM B RIGHT ANTI JOIN E ON a = x JOIN F ON x = z;\n"
    "M := SELECT YEAR(d) AS y, MONTH(d) AS m, DAY(d) AS dd, CAST_TO_INT(c) AS ci FROM B;\n"
    "N := FILTER B BY b LIKE \"x%y\" AND a != 3 OR a >= -4;\n",
    # catalog statements, sorted binary stores, DISTINCT
    "DESCRIBE t;\nSHOW TABLES;\nDROP TABLE t;\n"
    "STORE R INTO 'x' BINARY SORT SEGMENTS BY a;\n"
    "STORE R INTO 'x' BINARY PRESORTED BY a;\n"
    "P := SELECT DISTINCT a AS a, COUNT(a) AS c FROM B GROUP BY a;\n",
    # INSERT / DELETE queue their expressions; CASE sets a flag and queues nothing
    "INSERT INTO t SELECT a AS a, b*2 AS b FROM B;\n"
    "DELETE FROM t WHERE a > 5 AND b < 3;\n"
    "CREATE INDEX i1 ON t(a);\n"
    "Q := SELECT CASE WHEN a > 1 THEN b ELSE c END AS v FROM B;\n",
]
REJECTED = [
    "CREATE INTERVAL iv ON t(a, b);\n",  # bison.y:168, but fl.l has no INTERVAL token
    "X := SELECT a AS a FROM;\n",
]


def _engine_dump(script):
    L = ab.lib()
    L.alk_parse_dump.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]
    buf = ctypes.create_string_buffer(1 << 20)
    rc = L.alk_parse_dump(script.encode(), buf, len(buf))
    return rc, buf.value.decode()


def _reference_dump(script, tmp_path):
    p = tmp_path / "s.sql"
    p.write_text(script)
    r = subprocess.run([DUMP, str(p)], capture_output=True, text=True, timeout=60)
    return r.returncode, r.stdout


def test_operator_header_compiles_and_every_declaration_is_exported():
    subprocess.run(["g++", "-std=c++14", "-fsyntax-only", "-x", "c++", HDR], check=True)
    text = re.sub(r"/\*.*?\*/", "", open(HDR).read(), flags=re.S)
    funcs = set(re.findall(r"^\s*(?:void|int|size_t)\s+(\w+)\s*\(", text, flags=re.M))
    assert {"emit_select", "emit_filter", "emit_join", "emit_order", "emit_store", "emit_store_binary",
            "load_vars", "clean_queues", "alenkaExecute"} <= funcs
    nm = subprocess.run(["nm", "-DC", "--defined-only", ab.LIB_PATH], capture_output=True, text=True,
                        check=True).stdout
    exported = {ln.split(" ", 2)[2].split("(")[0] for ln in nm.splitlines() if len(ln.split(" ", 2)) == 3}
    missing = sorted(f for f in funcs if f not in exported)
    assert not missing, missing
    for g in ["op_type", "op_value", "op_nums", "op_nums_precision", "op_join", "join_type", "sel_count",
              "join_tab_cnt", "join_and_cnt", "varNames", "data_dict", "process_count", "hash_seed"]:
        assert any(e == g or e.startswith(g + "[") for e in exported), g


needs_frontend = pytest.mark.skipif(not os.path.exists(DUMP), reason="reference front end not built (oracle/ref.mk)")


@needs_frontend
@pytest.mark.parametrize("i", range(len(CORPUS)))
def test_reference_grammar_queues_what_the_engine_parser_queues(i, tmp_path):
    rc, want = _engine_dump(CORPUS[i])
    assert rc == 0, want
    rrc, got = _reference_dump(CORPUS[i], tmp_path)
    assert rrc == 0
    assert got == want


@needs_frontend
def test_golden_scripts_queue_identically(tmp_path):
    seen = set()
    for c in ref_cases.CASES:
        if c["script"] in seen:
            continue
        seen.add(c["script"])
        rc, want = _engine_dump(c["script"])
        assert rc == 0, (c["name"], want)
        rrc, got = _reference_dump(c["script"], tmp_path)
        assert rrc == 0 and got == want, c["name"]


@needs_frontend
@pytest.mark.parametrize("script", REJECTED)
def test_both_parsers_reject(script, tmp_path):
    rc, _ = _engine_dump(script)
    assert rc != 0
    rrc, out = _reference_dump(script, tmp_path)
    assert rrc != 0 and "PARSE ERROR" in out


CLI_CASES = ["flat_multi_q1_s1", "flat_multi_and_or_decimal", "flat_multi_zone_n_r_a", "three_way_q3_s1",
             "three_way_fused_decimal_all_groups", "three_way_join_alias_scale", "three_way_fused_never_dim",
             "config2_q3_s1"]


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(CLI), reason="reference front end not built (oracle/ref.mk)")
@pytest.mark.parametrize("name", CLI_CASES)
def test_reference_cli_on_the_engine_stores_the_reference_output(name, tmp_path_factory):
    case = gold.CASES[name]
    d = gold._dataset(case["dataset"], tmp_path_factory, gold._ProductGen)
    out = "cli_" + case["out"]
    script = case["script"].replace(f"'{case['out']}'", f"'{out}'")
    with open(os.path.join(d, "cli.sql"), "w") as f:
        f.write(script)
    p = os.path.join(d, out)
    if os.path.exists(p):
        os.remove(p)
    r = subprocess.run([CLI, "cli.sql"], cwd=d, capture_output=True, text=True, timeout=600)
    if "error" in case:  # process_error -> error_cb: printed, then exit(1) (callbacks.c:57-62)
        assert r.returncode == 1 and f"(Fatal) {case['error']}" in r.stdout, r.stdout[-500:]
        return
    assert r.returncode == 0, r.stdout[-500:] + r.stderr[-500:]
    gold._check(case, open(p, "rb").read())
