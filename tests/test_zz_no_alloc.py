"""alk_decode_segment_noalloc: the segment decode for callers that cannot call cudaMalloc
(a host that has handed all device memory to its own pools, or a decode path that must
not fail or stall on an allocation). It keeps its scan state in one fixed device array
instead of allocating, so these tests check, through the C ABI, that it returns exactly
what the allocating alk_decode_segment returns on two calls in a row (the shared array
still holds the previous call's state), and that it refuses segments above its stated
maximum. Integer results: compared bit for bit."""
import ctypes

import numpy as np
import pytest

import alenka_b200 as ab

pytestmark = pytest.mark.gpu

ALK_ERR_TOO_LARGE = 9
MAX_ROWS = 32768 * 2048


def _lib():
    L = ab.lib()
    sig = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int64, ctypes.c_int64,
           ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p]
    L.alk_decode_segment_noalloc.argtypes = sig
    L.alk_decode_segment.argtypes = sig
    L.alk_encode_segment.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_void_p,
                                     ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
    return L


def _segment(values, delta):
    """Encode values with the library's segment writer; return (meta, device payload)."""
    import torch
    L = _lib()
    values = np.ascontiguousarray(values, dtype=np.int64)
    cap = len(values) * 8 + 4096
    buf = ctypes.create_string_buffer(cap)
    ln = ctypes.c_size_t()
    assert L.alk_encode_segment(values.ctypes.data, len(values), int(delta), buf, cap, ctypes.byref(ln)) == 0
    img = buf.raw[:ln.value]
    cnt = int.from_bytes(img[0:4], "little")
    comp = int.from_bytes(img[20:24], "little")
    t = img[24 + cnt:]
    meta = dict(comp=comp, bits=int.from_bytes(t[8:12], "little"),
                lower=int.from_bytes(t[12:20], "little", signed=True), fit=int.from_bytes(t[20:24], "little"),
                start=int.from_bytes(t[24:32], "little", signed=True), rows=int.from_bytes(t[4:8], "little"))
    pad = np.zeros(((cnt + 255) // 256) * 256 + 256, dtype=np.uint8)
    pad[:cnt] = np.frombuffer(img[24:24 + cnt], dtype=np.uint8)
    return meta, torch.from_numpy(pad).cuda()


def _decode(fn, meta, payload):
    import torch
    out = torch.full((max(meta["rows"], 1),), -7, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    rc = fn(payload.data_ptr(), meta["comp"], meta["bits"], meta["fit"], meta["lower"], meta["start"], meta["rows"],
            out.data_ptr(), None)
    torch.cuda.synchronize()
    return rc, out.cpu().numpy()[:meta["rows"]]


def _inputs():
    rng = np.random.default_rng(2024)
    return [
        ("delta_multi_tile", np.cumsum(rng.integers(0, 50, 1_500_001)) - 10_000, True),
        ("delta_wide_gaps", np.cumsum(rng.integers(1, 1 << 30, 700_003)), True),
        ("delta_short", np.cumsum(rng.integers(0, 3, 1_000)), True),
        ("for_u16", rng.integers(0, 60_000, 300_000), False),
    ]


def test_noalloc_matches_allocating_decode_twice_in_a_row():
    L = _lib()
    for name, values, delta in _inputs():
        meta, payload = _segment(values, delta)
        assert meta["comp"] == (1 if delta else 0), name
        rc, want = _decode(L.alk_decode_segment, meta, payload)
        assert rc == 0 and np.array_equal(want, values), name
        for call in range(2):  # two calls in a row share the fixed scratch array
            rc, got = _decode(L.alk_decode_segment_noalloc, meta, payload)
            assert rc == 0, (name, call)
            assert np.array_equal(got, want), (name, call)


@pytest.mark.parametrize("rows", [MAX_ROWS + 1, 0xFFFFFFFF, 0xFFFFF801])
def test_noalloc_rejects_segments_above_its_maximum(rows):
    # 0xFFFFFFFF and 0xFFFFF801 would wrap a 32-bit tile count to 0; both must be refused
    import torch
    L = _lib()
    payload = torch.zeros(4096, dtype=torch.uint8, device="cuda")
    out = torch.full((8,), -7, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    rc = L.alk_decode_segment_noalloc(payload.data_ptr(), 1, 2, 32, 0, 0, rows, out.data_ptr(), None)
    torch.cuda.synchronize()
    assert rc == ALK_ERR_TOO_LARGE
    assert (out.cpu().numpy() == -7).all()


def test_noalloc_accepts_exactly_its_maximum_and_allocates_nothing():
    """MAX_ROWS rows of a 1-bit FOR-delta segment (an 8 MB payload, a 512 MB output):
    accepted and decoded exactly, twice, with the device's free memory unchanged across
    the warm calls."""
    import torch
    L = _lib()
    rng = np.random.default_rng(77)
    steps = rng.integers(0, 2, MAX_ROWS, dtype=np.int64)
    steps[0] = 0
    values = np.cumsum(steps) + 1000
    meta, payload = _segment(values, True)
    assert meta["comp"] == 1 and meta["bits"] == 1 and meta["rows"] == MAX_ROWS
    out = torch.full((MAX_ROWS,), -7, dtype=torch.int64, device="cuda")
    args = (payload.data_ptr(), meta["comp"], meta["bits"], meta["fit"], meta["lower"], meta["start"],
            meta["rows"], out.data_ptr(), None)
    assert L.alk_decode_segment_noalloc(*args) == 0  # first call: looks up the array's address
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for call in range(2):
        out.fill_(-7)
        torch.cuda.synchronize()
        assert L.alk_decode_segment_noalloc(*args) == 0, call
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free_before, call
        assert np.array_equal(out.cpu().numpy(), values), call
