"""Golden vectors produced by the reference's own code (tests/golden/make_golden.sh):
segment files written by the reference's pfor_compress / pfor_delta_compress and
MurmurHash64A values. They pin the oracle's decoder and hash, the product's segment
writer, and (GPU) the product's decode kernels."""
import ctypes
import glob
import os

import numpy as np
import pytest

import alenka_b200 as ab

from . import _oracle
from .test_cpu import _py_murmur

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLD, "ref_codec", "*.seg")))


def _case(name):
    seg = open(os.path.join(GOLD, "ref_codec", name + ".seg"), "rb").read()
    vals = np.fromfile(os.path.join(GOLD, "ref_codec", name + ".values"), dtype=np.int64)
    return seg, vals


def test_golden_cases_present():
    assert len(CASES) == 11


@pytest.mark.parametrize("name", CASES)
def test_oracle_decodes_reference_segments(name):
    seg, vals = _case(name)
    buf = ctypes.create_string_buffer(seg, len(seg))
    out = np.zeros(len(vals) + 1, dtype=np.int64)
    n = _oracle.lib().oracle_decode_segment(buf, len(seg), out.ctypes.data, out.size)
    assert n == len(vals)
    assert np.array_equal(out[:n], vals)


@pytest.mark.parametrize("name", CASES)
def test_writer_matches_reference_bytes(name):
    seg, vals = _case(name)
    L = ab.lib()
    L.alk_encode_segment.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_void_p,
                                     ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
    out = ctypes.create_string_buffer(len(seg) + 4096)
    ln = ctypes.c_size_t()
    delta = 1 if name.startswith("delta") else 0
    rc = L.alk_encode_segment(vals.ctypes.data, len(vals), delta, out, len(out), ctypes.byref(ln))
    assert rc == 0
    assert out.raw[:ln.value] == seg


def test_murmur_golden():
    lines = open(os.path.join(GOLD, "murmur64a.txt")).read().split("\n")
    n = 0
    for ln in lines:
        if not ln:
            continue
        seed, hexb, h = ln.split(" ")
        data = b"" if hexb == "-" else bytes.fromhex(hexb)
        assert _oracle.murmur64a(data, int(seed)) == int(h)
        assert _py_murmur(data, int(seed)) == int(h)
        n += 1
    assert n == 123


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_gpu_decode_matches_reference(name):
    import torch
    seg, vals = _case(name)
    cnt = int.from_bytes(seg[0:4], "little")
    comp = int.from_bytes(seg[20:24], "little")
    t = seg[24 + cnt:]
    rec, bits = int.from_bytes(t[4:8], "little"), int.from_bytes(t[8:12], "little")
    lower = int.from_bytes(t[12:20], "little", signed=True)
    fit = int.from_bytes(t[20:24], "little")
    start = int.from_bytes(t[24:32], "little", signed=True)
    payload = np.frombuffer(seg[24:24 + cnt], dtype=np.uint8)
    pad = np.zeros(((cnt + 255) // 256) * 256 + 256, dtype=np.uint8)
    pad[:cnt] = payload
    d_pay = torch.from_numpy(pad).cuda()
    d_out = torch.zeros(max(rec, 1), dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    rc = ab.lib().alk_decode_segment(d_pay.data_ptr(), comp, bits, fit, lower, start, rec, d_out.data_ptr(), None)
    torch.cuda.synchronize()
    assert rc == 0
    assert np.array_equal(d_out.cpu().numpy()[:rec], vals)


def like_golden():
    """(width, entries as bytes, [(pattern bytes, [0/1 per entry])]) written by the
    reference's own LIKE matcher (gpu_regex, filter.cu:67-129) via make_golden.sh."""
    width, entries, cases = 0, [], []
    for ln in open(os.path.join(GOLD, "like_gpu_regex.txt")).read().splitlines():
        f = ln.split()
        if f[0] == "width":
            width = int(f[1])
        elif f[0] == "entry":
            entries.append(bytes.fromhex(f[1]))
        elif f[0] == "pattern":
            pat = b"" if f[1] == "-" else bytes.fromhex(f[1])
            cases.append((pat, [int(c) for c in f[2]]))
    return width, entries, cases


def test_oracle_like_matches_reference():
    width, entries, cases = like_golden()
    assert width == 12 and len(entries) == 22 and len(cases) == 40
    L = _oracle.lib()
    L.oracle_like.argtypes = [ctypes.c_char_p, ctypes.c_uint32, ctypes.c_char_p]
    for pat, want in cases:
        got = [L.oracle_like(e, width, pat + b"\0") for e in entries]
        assert got == want, pat
