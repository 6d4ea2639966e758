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
