"""LIKE on char columns: the dictionary matcher on the device against the reference's own
matcher (golden vectors from gpu_regex, filter.cu:67-129), and whole scripts with LIKE
filters against the oracle, byte for byte, on the operator path and the fused plans."""
import ctypes
import os

import numpy as np
import pytest

import alenka_b200 as ab
from alenka_b200 import workloads as wl

from . import _oracle
from .test_golden import like_golden
from .test_gpu_parity import _read

pytestmark = pytest.mark.gpu


def test_device_matcher_matches_reference():
    import torch
    width, entries, cases = like_golden()
    L = ab.lib()
    L.alk_like_dictionary.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_char_p,
                                      ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p]
    d_dict = torch.from_numpy(np.frombuffer(b"".join(entries), dtype=np.uint8).copy()).cuda()
    for pat, want in cases:
        d_bits = torch.full((1 + (len(entries) + 31) // 32,), -1, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        assert L.alk_like_dictionary(d_dict.data_ptr(), width, len(entries), pat, len(pat), d_bits.data_ptr(),
                                     None) == 0
        torch.cuda.synchronize()
        words = d_bits.cpu().numpy().view(np.uint32)
        assert words[0] == len(entries)
        got = [int(words[1 + k // 32] >> (k % 32) & 1) for k in range(len(entries))]
        assert got == want, pat


PATTERNS = ["%", "%%", "", "A%", "%A", "%A%", "A?B", "???", "?%", "%?", "%.%", "%B%X%", "AB", "A_B%",
            "%_%", "X%X", "%XX", "?.?", "A%B%", "%AB", "A%%B", "%\\%", "B%%%", "%?%?%?%?", "%.", ".%",
            "A?.%", "%B_", "XXXXXXXXXXX", "%BA%AB%"]


@pytest.fixture(scope="module")
def names(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("names"))
    ab.gen_names(d, 200_000, 2_000, 60_000, 9)
    return d


def _both(d, script, out):
    _oracle.execute(d, script.replace(out, "oracle_" + out))
    want = _read(os.path.join(d, "oracle_" + out))
    got = {}
    for plain in (False, True):
        with ab.Session(d, plain=plain) as s:
            s.execute(script)
        got[plain] = _read(os.path.join(d, out))
    return want, got


@pytest.mark.parametrize("pat", PATTERNS)
def test_like_filter_group_by_matches_oracle(names, pat):
    script = (f'NF := FILTER names BY n_name LIKE "{pat}";\n'
              "R := SELECT n_name AS nm, COUNT(n_key) AS c, SUM(n_key) AS s FROM NF GROUP BY n_name;\n"
              "STORE R INTO 'like.txt' USING ('|');\n")
    want, got = _both(names, script, "like.txt")
    assert got[False] == want and got[True] == want


def test_like_combined_with_other_predicates(names):
    script = ('NF := FILTER names BY (n_name LIKE "A%" AND n_key > 50000) OR n_name LIKE "%.%X";\n'
              "R := SELECT n_key AS k, n_name AS nm FROM NF;\n"
              "STORE R INTO 'likec.txt' USING ('|');\n")
    want, got = _both(names, script, "likec.txt")
    assert got[False] == want and got[True] == want and want


def test_like_in_the_fused_three_way_plan(tmp_path):
    """The customer build stage filtered by LIKE on c_mktsegment (width 10, where
    AUTOMOBILE fills the width and has no terminator)."""
    d = str(tmp_path)
    wl.make_three_way(d, scale=0.002, seg_rows=50_000, seed=4)
    base = wl.three_way_script(4, out="tw.txt")
    lines = base.split("\n")
    k = next(i for i, ln in enumerate(lines) if "c_mktsegment" in ln)
    for pat in ("%I%", "AUTOMOBILE", "AUTOMOBILE%", "%E", "M?CHINERY", "%O%O%"):
        lines[k] = f'CF := FILTER customer BY c_mktsegment LIKE "{pat}";'
        script = "\n".join(lines)
        want, got = _both(d, script, "tw.txt")
        assert got[False] == want and got[True] == want, pat
        with ab.Session(d) as s:
            s.execute(script)
            assert s.stats().plan != 0  # a fused plan ran
