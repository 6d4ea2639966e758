"""The text loader (LOAD ... USING (sep) AS (...)) against the reference's own: the golden
digests in tests/golden/text_load.json come from the reference CLI built for the CPU
(tests/golden/make_text_load.py). CPU: the case files are unchanged; where the reference
build is present, the oracle restatement (oracle/textload.py) equals the values the
reference stored. GPU: the engine's LOAD + STORE BINARY writes the same segment and
header files, byte for byte, and the query over them stores the same rows."""
import hashlib
import json
import os
import re
import struct
import subprocess

import numpy as np
import pytest

from . import text_cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = json.load(open(os.path.join(ROOT, "tests", "golden", "text_load.json")))
REF = os.path.join(ROOT, "oracle", "_ref", "alenka_ref")


def _sha(b):
    return hashlib.sha256(b).hexdigest()


def _write_case(d, name):
    text = text_cases.CASES[name]["text"]().encode()
    with open(os.path.join(d, text_cases.FILES[name]), "wb") as f:
        f.write(text)
    return text


@pytest.mark.parametrize("name", sorted(text_cases.CASES))
def test_case_files_unchanged(name):
    assert _sha(text_cases.CASES[name]["text"]().encode()) == GOLD[name]["text_sha256"]


def _for_values(path):
    """Values of a FOR segment file (header, payload at its width, trailer)."""
    b = open(path, "rb").read()
    cnt = struct.unpack_from("<I", b, 0)[0]
    comp = struct.unpack_from("<I", b, 20)[0]
    assert comp == 0
    tail = 24 + cnt
    n, bits, lower = struct.unpack_from("<IIq", b, tail + 4)
    dt = {8: np.uint8, 16: np.uint16, 32: np.uint32, 64: np.uint64}[bits]
    raw = np.frombuffer(b, dtype=dt, count=n, offset=24).astype(np.uint64)
    return ((raw + np.uint64(lower & (2**64 - 1))).astype(np.uint64).view(np.int64)).tolist()


@pytest.mark.skipif(not os.path.exists(REF), reason="reference build absent (oracle/build_ref.sh)")
@pytest.mark.parametrize("name", sorted(text_cases.CASES))
def test_oracle_restatement_equals_the_reference(name, tmp_path):
    from oracle import textload
    case = text_cases.CASES[name]
    d = str(tmp_path)
    text = _write_case(d, name)
    with open(os.path.join(d, "s.sql"), "w") as f:
        f.write(case["scripts"][0])
    subprocess.run([REF, "s.sql"], cwd=d, capture_output=True, timeout=600, check=True)
    m = re.search(r"AS \((.*)\);", case["scripts"][0])
    cols, names = [], []
    for part in m.group(1).split(", "):
        nm, rest = part.split("{")
        field, ty = rest.split("}:")
        if ty.startswith("decimal"):
            kind, scale = "decimal", int(ty.split(",")[1].rstrip(")"))
        elif ty.startswith("varchar"):
            kind, scale = "char", int(ty.split("(")[1].split(")")[0])
        else:
            kind, scale = "int", 0
        cols.append((int(field), kind, scale))
        names.append(nm)
    got = textload.load(text, "|", cols)
    for (_, kind, w), nm, vals in zip(cols, names, got):
        p = os.path.join(d, f"{case['table']}.{nm}")
        if kind != "char":
            assert _for_values(p + ".0") == vals, nm
            continue
        # char: the dictionary's values at the stored codes (NO ENCODING codes count from 1)
        dic = open(p, "rb").read()
        codes = _for_values(p + ".0.idx")
        base = 1 if "NO ENCODING" in case["scripts"][0].split(nm + "{")[1].split(",")[0] else 0
        assert [dic[(c - base) * w:(c - base + 1) * w] for c in codes] == vals, nm


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(text_cases.CASES))
def test_engine_load_and_store_binary_match_the_reference(name, tmp_path):
    import alenka_b200 as ab
    case = text_cases.CASES[name]
    d = str(tmp_path)
    _write_case(d, name)
    for script in case["scripts"]:
        with ab.Session(d) as s:
            s.execute(script)
    for fn, digest in GOLD[name]["files"].items():
        assert _sha(open(os.path.join(d, fn), "rb").read()) == digest, fn


def test_records_are_newline_terminated_lines():
    from oracle import textload
    text = b"1|2|\n3|4|\n5|6"
    assert textload.load(text, "|", [(1, "int", 0), (2, "int", 0)]) == [[1, 3], [2, 4]]


@pytest.mark.gpu
def test_join_on_char_keys_of_two_dictionaries(tmp_path):
    """A string-key join between tables whose char columns have different dictionaries
    (different names, widths 25 and 20, values first seen in different orders): the
    engine compares the values (MurmurHash64A of each value padded to the wider width)
    where the reference would compare the two dictionaries' codes. Checked against the
    join computed by string equality."""
    import random
    import alenka_b200 as ab
    d = str(tmp_path)
    r = random.Random(5)
    alnum = "ABCDEFGHIJKLMNOPQRSTUVWXYZ0123456789"
    names = ["".join(r.choice(alnum) for _ in range(r.randint(4, 20))) for _ in range(800)]
    names = sorted(set(names))
    segs = {n: r.choice(["AUTO", "BUILD", "FURN"]) for n in names}
    cust = list(names)
    r.shuffle(cust)
    with open(os.path.join(d, "cust.tbl"), "w") as f:
        for n in cust:
            f.write(f"{n}|{segs[n]}|\n")
    orders = []
    with open(os.path.join(d, "ord.tbl"), "w") as f:
        for i in range(6000):
            n = r.choice(names) if r.random() < 0.9 else "NOPE" + str(i % 7)
            amt = r.randint(1, 1000)
            orders.append((n, amt))
            f.write(f"{i}|{n}|{amt}|\n")
    with ab.Session(d) as s:
        s.execute("C := LOAD 'cust.tbl' USING ('|') AS (c_name{1}:varchar(25), c_seg{2}:varchar(8));\n"
                  "STORE C INTO 'cust' BINARY;\n"
                  "O := LOAD 'ord.tbl' USING ('|') AS (o_id{1}:int, o_cname{2}:varchar(20), o_amt{3}:int);\n"
                  "STORE O INTO 'ord' BINARY;\n")
    with ab.Session(d) as s:
        s.execute("J := SELECT c_seg AS seg, o_amt AS amt FROM ord JOIN cust ON o_cname = c_name;\n"
                  "R := SELECT seg AS seg, SUM(amt) AS s, COUNT(amt) AS c FROM J GROUP BY seg;\n"
                  "STORE R INTO 'j.txt' USING ('|');\n")
    got = set()
    for line in open(os.path.join(d, "j.txt"), "rb").read().decode().splitlines():
        seg, sm, cnt = line.split("|")[:3]
        got.add((seg.rstrip("\x00"), int(sm), int(cnt)))
    want = {}
    for n, amt in orders:
        if n in segs:
            k = segs[n]
            s_, c_ = want.get(k, (0, 0))
            want[k] = (s_ + amt, c_ + 1)
    assert got == {(k, v[0], v[1]) for k, v in want.items()}
