"""Segment writer on the GPU (alk_encode_segment_device) against the reference's own
segment files and the host writer, byte for byte.

The reference writes a column segment with pfor_compress / pfor_delta_compress
(compress.cu:271-527); tests/golden/ref_codec holds files that it wrote. The device
writer must produce the same bytes for the same values, and the same bytes as the host
writer (alk_encode_segment, pinned to those files in test_golden.py) on every other
input. Images are also decoded by the oracle's decoder (a round trip)."""
import ctypes
import os

import numpy as np
import pytest

import alenka_b200 as ab

from . import _oracle
from .test_golden import CASES, _case

pytestmark = pytest.mark.gpu


def _declare():
    L = ab.lib()
    L.alk_encode_segment_device.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_void_p,
                                            ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t), ctypes.c_void_p]
    L.alk_encode_segment.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_void_p,
                                     ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
    return L


def device_image(vals, mode, cap=None):
    """(status, image bytes) of the device writer for int64 numpy values."""
    import torch
    L = _declare()
    n = len(vals)
    d_v = torch.from_numpy(np.ascontiguousarray(vals, dtype=np.int64)).cuda() if n else \
        torch.zeros(1, dtype=torch.int64, device="cuda")
    cap = 24 + 8 * n + 32 + 8 if cap is None else cap
    d_img = torch.full((max(cap, 8) // 8 + 1,), -1, dtype=torch.int64, device="cuda")  # 8-byte aligned
    ln = ctypes.c_size_t()
    torch.cuda.synchronize()
    rc = L.alk_encode_segment_device(d_v.data_ptr(), n, mode, d_img.data_ptr(), cap, ctypes.byref(ln), None)
    torch.cuda.synchronize()
    if rc:
        return rc, ln.value
    return 0, d_img.cpu().numpy().view(np.uint8)[:ln.value].tobytes()


def host_image(vals, delta):
    L = _declare()
    v = np.ascontiguousarray(vals, dtype=np.int64)
    out = ctypes.create_string_buffer(24 + 8 * len(v) + 64)
    ln = ctypes.c_size_t()
    assert L.alk_encode_segment(v.ctypes.data, len(v), delta, out, len(out), ctypes.byref(ln)) == 0
    return out.raw[:ln.value]


def oracle_decode(img):
    buf = ctypes.create_string_buffer(img, len(img))
    rec = int.from_bytes(img[-28:-24], "little")
    out = np.zeros(rec + 1, dtype=np.int64)
    n = _oracle.lib().oracle_decode_segment(buf, len(img), out.ctypes.data, out.size)
    return out[:n]


@pytest.mark.parametrize("name", CASES)
def test_device_writer_matches_reference_files(name):
    seg, vals = _case(name)
    mode = 2 if name.startswith("delta") else 0  # the reference's delta switch: delta when sorted
    rc, img = device_image(vals, mode)
    assert rc == 0
    assert img == seg


def _inputs():
    r = np.random.default_rng(11)
    out = []
    for n in (1, 2, 3, 7, 8, 9, 31, 33, 1000, 4097, 65_537, 1_000_003):
        out.append(("u8", r.integers(-50, 200, n)))
        out.append(("u16", r.integers(19_920_101, 19_981_231, n)))
        out.append(("u32", r.integers(-(1 << 30), 1 << 30, n)))
        out.append(("u64", r.integers(-(1 << 62), 1 << 62, n)))
        out.append(("const", np.full(n, -7)))
        out.append(("sorted_small", np.cumsum(r.integers(0, 5, n)) + 1000))
        out.append(("sorted_wide", np.cumsum(r.integers(0, 1 << 40, n)) - (1 << 50)))
        out.append(("sorted_dups", np.cumsum(r.integers(0, 2, n) * 4)))
    out.append(("extremes", np.array([np.iinfo(np.int64).min, 0, np.iinfo(np.int64).max] * 5)))
    return out


@pytest.mark.parametrize("mode", [0, 2])
def test_device_writer_matches_host_writer(mode):
    for name, v in _inputs():
        rc, img = device_image(v, mode)
        assert rc == 0, name
        assert img == host_image(v, 1 if mode == 2 else 0), (name, len(v))
        if name != "extremes":  # a span above 2^63 has no width in the format
            assert np.array_equal(oracle_decode(img), v), (name, len(v))


def test_forced_delta_round_trips_unsorted_values():
    r = np.random.default_rng(5)
    for n in (1, 2, 100, 99_999):
        v = r.integers(-(1 << 40), 1 << 40, n)
        rc, img = device_image(v, 1)
        assert rc == 0
        assert int.from_bytes(img[20:24], "little") == 1  # comp_type FOR-delta
        assert np.array_equal(oracle_decode(img), v)


def test_empty_segment_matches_host_frame():
    rc, img = device_image(np.zeros(0, np.int64), 0)
    assert rc == 0 and len(img) == 56
    assert int.from_bytes(img[0:4], "little") == 0  # no payload


def test_capacity_and_arguments():
    import torch
    L = _declare()
    v = np.arange(1000, dtype=np.int64) * 3
    rc, need = device_image(v, 0, cap=100)
    assert rc == 3 and need == 24 + 2000 + 32  # ALK_ERR_OVERFLOW with the exact size: 16-bit FOR
    rc, img = device_image(v, 0, cap=need)
    assert rc == 0 and len(img) == need
    d_v = torch.from_numpy(v).cuda()
    d_img = torch.zeros(1024, dtype=torch.int64, device="cuda")
    ln = ctypes.c_size_t()
    assert L.alk_encode_segment_device(d_v.data_ptr() + 4, 10, 0, d_img.data_ptr(), 8192, ctypes.byref(ln),
                                       None) == 1  # misaligned values
    assert L.alk_encode_segment_device(d_v.data_ptr(), 10, 3, d_img.data_ptr(), 8192, ctypes.byref(ln),
                                       None) == 1  # no such mode


def test_large_segment_round_trip_on_device():
    """60M values (a lineitem column's worth): the device image decodes, on the device,
    back to the values, and equals the host writer's image."""
    import torch
    L = ab.lib()
    n = 60_000_000
    r = np.random.default_rng(3)
    v = r.integers(90_000, 10_500_000, n)
    rc, img = device_image(v, 0)
    assert rc == 0
    assert img == host_image(v, 0)
    cnt = int.from_bytes(img[0:4], "little")
    t = img[24 + cnt:]
    bits = int.from_bytes(t[8:12], "little")
    lower = int.from_bytes(t[12:20], "little", signed=True)
    pad = np.zeros(cnt + 256, dtype=np.uint8)
    pad[:cnt] = np.frombuffer(img[24:24 + cnt], dtype=np.uint8)
    d_pay = torch.from_numpy(pad).cuda()
    d_out = torch.zeros(n, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    assert L.alk_decode_segment(d_pay.data_ptr(), 0, bits, 64 // bits, lower, 0, n, d_out.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert torch.equal(d_out.cpu(), torch.from_numpy(v))


def batch_images(arrays, mode):
    """(status, [image bytes]) of the batched device writer over numpy int64 arrays."""
    import torch
    L = ab.lib()
    vp = ctypes.c_void_p
    L.alk_encode_segments_device.argtypes = [vp, vp, ctypes.c_uint32, ctypes.c_int, vp, vp, vp, vp]
    k = len(arrays)
    d_vals = [torch.from_numpy(np.ascontiguousarray(a, dtype=np.int64)).cuda() if len(a) else
              torch.zeros(1, dtype=torch.int64, device="cuda") for a in arrays]
    caps = [24 + 8 * len(a) + 32 for a in arrays]
    d_imgs = [torch.full((c // 8 + 2,), -1, dtype=torch.int64, device="cuda") for c in caps]
    P = ctypes.c_void_p * k
    ptrs = P(*[t.data_ptr() for t in d_vals])
    imgs = P(*[t.data_ptr() for t in d_imgs])
    ns = (ctypes.c_uint32 * k)(*[len(a) for a in arrays])
    cp = (ctypes.c_size_t * k)(*caps)
    lens = (ctypes.c_size_t * k)()
    torch.cuda.synchronize()
    rc = L.alk_encode_segments_device(ptrs, ns, k, mode, imgs, cp, lens, None)
    torch.cuda.synchronize()
    if rc:
        return rc, list(lens)
    return 0, [d_imgs[i].cpu().numpy().view(np.uint8)[:lens[i]].tobytes() for i in range(k)]


def _edge_ranges():
    """Value and difference ranges at and around every power of two: the batched plan
    computes widths exactly up to 2^46 and leaves the rest to the single-segment path."""
    out = []
    for kk in range(1, 63):
        for span in (1 << kk) - 1, 1 << kk, (1 << kk) + 1:
            out.append(np.array([0, span - 1], dtype=np.int64))          # value range: span
            out.append(np.array([5, 5, 5 + span - 1], dtype=np.int64))   # difference range: span
    return out


@pytest.mark.parametrize("mode", [0, 2])
def test_batched_writer_matches_host_writer(mode):
    inputs = [v for _, v in _inputs()] + [np.zeros(0, np.int64)] + _edge_ranges()
    for name, v in _reference_values():
        inputs.append(v)
    rc, imgs = batch_images(inputs, mode)
    assert rc == 0
    for v, img in zip(inputs, imgs):
        if len(v) == 0:
            assert len(img) == 56
            continue
        assert img == host_image(v, 1 if mode == 2 else 0), len(v)


def _reference_values():
    return [(name, _case(name)[1]) for name in CASES]


def test_batched_writer_reference_files_and_forced_delta():
    seg = {name: _case(name) for name in CASES}
    rc, imgs = batch_images([seg[n][1] for n in CASES], 2)
    assert rc == 0
    for n, img in zip(CASES, imgs):
        if n.startswith("delta"):
            assert img == seg[n][0], n
    r = np.random.default_rng(8)
    vals = [r.integers(-(1 << 40), 1 << 40, n) for n in (1, 2, 3, 8191, 8192, 8193, 50_000)]
    rc, imgs = batch_images(vals, 1)
    assert rc == 0
    for v, img in zip(vals, imgs):
        assert np.array_equal(oracle_decode(img), v)


def test_batched_writer_needs_room_for_the_largest_image():
    import torch
    L = ab.lib()
    vp = ctypes.c_void_p
    L.alk_encode_segments_device.argtypes = [vp, vp, ctypes.c_uint32, ctypes.c_int, vp, vp, vp, vp]
    d_v = torch.arange(100, dtype=torch.int64, device="cuda")
    d_img = torch.zeros(256, dtype=torch.int64, device="cuda")
    ptrs = (ctypes.c_void_p * 1)(d_v.data_ptr())
    imgs = (ctypes.c_void_p * 1)(d_img.data_ptr())
    ns = (ctypes.c_uint32 * 1)(100)
    cp = (ctypes.c_size_t * 1)(24 + 100 + 32)  # the FOR image would fit, the largest would not
    lens = (ctypes.c_size_t * 1)()
    assert L.alk_encode_segments_device(ptrs, ns, 1, 0, imgs, cp, lens, None) == 3
    assert lens[0] == 24 + 800 + 32
