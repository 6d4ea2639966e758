"""Fused-stage entry points through the C ABI, checked against numpy on the same inputs:
the build stage's survivor list (overflow applies nothing and reports the exact survivor
count; a rerun with that count succeeds), the asynchronous status form, the exact key
bitmap under a key range, and the device-side top-k selection and row gather (ties
included). Integer results: compared exactly."""
import ctypes as c

import numpy as np
import pytest

import alenka_b200 as ab

pytestmark = pytest.mark.gpu

ALK_OK, ALK_ERR_OVERFLOW = 0, 3


class ColSeg(c.Structure):
    _fields_ = [("data", c.c_void_p), ("lower", c.c_int64), ("rows", c.c_uint32), ("bits", c.c_uint32)]


class StageStatus(c.Structure):
    _fields_ = [("rows_in", c.c_uint64), ("reserved", c.c_uint64), ("err", c.c_int32), ("pad", c.c_int32),
                ("hits", c.c_uint64)]


class HtStatus(c.Structure):
    _fields_ = [("inserted", c.c_uint64), ("flags", c.c_int32 * 4)]


def _lib():
    L = ab.lib()
    vp, u32, u64, i32, i64 = c.c_void_p, c.c_uint32, c.c_uint64, c.c_int32, c.c_int64
    L.alk_ht_create_range.argtypes = [u64, u32, i64, i64, c.POINTER(vp), vp]
    L.alk_ht_free.argtypes = [vp, vp]
    L.alk_ht_free.restype = None
    L.alk_ht_info.argtypes = [vp, c.POINTER(u64), c.POINTER(c.c_int), vp]
    L.alk_ht_info_async.argtypes = [vp, c.POINTER(HtStatus), vp]
    L.alk_ht_slots.argtypes = [vp]
    L.alk_ht_slots.restype = u64
    L.alk_ht_payload.argtypes = [vp, u32]
    L.alk_ht_payload.restype = vp
    L.alk_ht_keys.argtypes = [vp]
    L.alk_ht_keys.restype = vp
    L.alk_pipeline_build.argtypes = [c.POINTER(ColSeg), u32, u32, c.POINTER(c.c_uint8), vp, vp, i32, vp, i32,
                                     c.POINTER(i32), u64, c.POINTER(u64), c.POINTER(u64), vp]
    L.alk_pipeline_build_async.argtypes = [c.POINTER(ColSeg), u32, u32, c.POINTER(c.c_uint8), vp, vp, i32, vp, i32,
                                           c.POINTER(i32), u64, c.POINTER(StageStatus), vp]
    L.alk_topk_select.argtypes = [vp, vp, u64, u32, vp, u64, vp, vp]
    L.alk_gather_rows.argtypes = [c.POINTER(vp), u32, vp, vp, u64, vp, vp]
    return L


def _column(values, bits=32):
    """A FOR column segment on the device: stored = value - min, at `bits` width, padded."""
    import torch
    lo = int(values.min())
    dt = {8: np.uint8, 16: np.uint16, 32: np.uint32, 64: np.uint64}[bits]
    raw = (values - lo).astype(dt)
    pad = np.zeros(len(raw) * raw.itemsize + 256, dtype=np.uint8)
    pad[:len(raw) * raw.itemsize] = raw.view(np.uint8)
    t = torch.from_numpy(pad).cuda()
    return t, ColSeg(t.data_ptr(), lo, len(values), bits)


def test_build_hit_list_overflow_then_exact_rerun():
    # a predicate that is not a conjunction runs on the register-machine scan, which
    # hands its survivors to the hit kernel through the survivor list
    import torch
    L = _lib()
    n = 2_000_000
    keys = np.random.default_rng(3).permutation(n).astype(np.int64) * 3 + 11
    buf, cs = _column(keys)
    cols = (ColSeg * 1)(cs)
    mode = (c.c_uint8 * 1)(2)
    pred = _or_pred(0, 0)  # key >= 0 OR key < 0: every row
    ht = c.c_void_p()
    assert L.alk_ht_create_range(n, 0, int(keys.min()), int(keys.max()), c.byref(ht), None) == ALK_OK
    try:
        rows_in, hits = c.c_uint64(), c.c_uint64()
        rc = L.alk_pipeline_build(cols, 1, 1, mode, c.byref(pred), None, -1, ht, 0, None, 1, c.byref(rows_in),
                                  c.byref(hits), None)
        assert rc == ALK_ERR_OVERFLOW
        assert hits.value == n and rows_in.value == n
        ins, fl = c.c_uint64(), c.c_int()
        assert L.alk_ht_info(ht, c.byref(ins), c.byref(fl), None) == ALK_OK
        assert ins.value == 0 and fl.value == 0  # nothing applied
        rc = L.alk_pipeline_build(cols, 1, 1, mode, c.byref(pred), None, -1, ht, 0, None, hits.value,
                                  c.byref(rows_in), c.byref(hits), None)
        assert rc == ALK_OK and hits.value == n
        assert L.alk_ht_info(ht, c.byref(ins), c.byref(fl), None) == ALK_OK
        assert ins.value == n and fl.value == 0
    finally:
        L.alk_ht_free(ht, None)
        torch.cuda.synchronize()
    del buf


def test_build_inline_from_staged_tile():
    # no predicate and no probe: the TMA-staged scan inserts its rows itself (no survivor
    # list, so no list capacity applies); a duplicate key is reported
    import torch
    L = _lib()
    n = 2_000_000
    keys = np.random.default_rng(4).permutation(n).astype(np.int64) * 3 + 11
    buf, cs = _column(keys)
    cols = (ColSeg * 1)(cs)
    mode = (c.c_uint8 * 1)(2)
    ht = c.c_void_p()
    assert L.alk_ht_create_range(n, 0, int(keys.min()), int(keys.max()), c.byref(ht), None) == ALK_OK
    try:
        rows_in, hits = c.c_uint64(), c.c_uint64()
        rc = L.alk_pipeline_build(cols, 1, 1, mode, None, None, -1, ht, 0, None, 1, c.byref(rows_in), c.byref(hits),
                                  None)
        assert rc == ALK_OK and rows_in.value == n
        ins, fl = c.c_uint64(), c.c_int()
        assert L.alk_ht_info(ht, c.byref(ins), c.byref(fl), None) == ALK_OK
        assert ins.value == n and fl.value == 0
        # the same keys again: every insert meets its duplicate
        rc = L.alk_pipeline_build(cols, 1, 1, mode, None, None, -1, ht, 0, None, 0, c.byref(rows_in), c.byref(hits),
                                  None)
        assert rc == ALK_OK
        assert L.alk_ht_info(ht, c.byref(ins), c.byref(fl), None) == ALK_OK
        assert ins.value == n and (fl.value & 1)
    finally:
        L.alk_ht_free(ht, None)
        torch.cuda.synchronize()
    del buf


class Instr(c.Structure):
    _fields_ = [("op", c.c_uint8), ("dst", c.c_uint8), ("ka", c.c_uint8), ("kb", c.c_uint8), ("a", c.c_uint16),
                ("b", c.c_uint16), ("pad", c.c_uint32)]


class Program(c.Structure):
    _fields_ = [("n_instr", c.c_uint32), ("result", c.c_uint32), ("ins", Instr * 48), ("consts", c.c_int64 * 48)]


ALK_OP_LT, ALK_OP_GE, ALK_OP_AND = 5, 8, 11
ALK_K_REG, ALK_K_COL, ALK_K_CONST = 0, 1, 2


def _range_pred(slot, lo, hi):
    """lo <= column(slot) < hi as a compiled program (two conjuncts)."""
    p = Program()
    p.n_instr, p.result = 3, 2
    p.consts[0], p.consts[1] = lo, hi
    p.ins[0] = Instr(ALK_OP_GE, 0, ALK_K_COL, ALK_K_CONST, slot, 0, 0)
    p.ins[1] = Instr(ALK_OP_LT, 1, ALK_K_COL, ALK_K_CONST, slot, 1, 0)
    p.ins[2] = Instr(ALK_OP_AND, 2, ALK_K_REG, ALK_K_REG, 0, 1, 0)
    return p


ALK_OP_OR = 12


def _or_pred(slot, c0):
    """column(slot) >= c0 OR column(slot) < c0 (true for every row; not a conjunction)."""
    p = Program()
    p.n_instr, p.result = 3, 2
    p.consts[0] = c0
    p.ins[0] = Instr(ALK_OP_GE, 0, ALK_K_COL, ALK_K_CONST, slot, 0, 0)
    p.ins[1] = Instr(ALK_OP_LT, 1, ALK_K_COL, ALK_K_CONST, slot, 0, 0)
    p.ins[2] = Instr(ALK_OP_OR, 2, ALK_K_REG, ALK_K_REG, 0, 1, 0)
    return p


@pytest.mark.parametrize("bits", [16, 32, 64])
def test_build_async_status_and_payload(bits):
    import torch
    L = _lib()
    rng = np.random.default_rng(5)
    n = 300_000
    keys = rng.permutation(n).astype(np.int64) + 1000
    vals = rng.integers(-20_000, 40_000, n).astype(np.int64)
    kb, ks = _column(keys)
    vb, vs = _column(vals, bits)
    cols = (ColSeg * 2)(ks, vs)
    mode = (c.c_uint8 * 1)(2)
    prog = _range_pred(1, -5_000, 30_000)
    sel = (vals >= -5_000) & (vals < 30_000)
    ht = c.c_void_p()
    assert L.alk_ht_create_range(n, 1, 1000, 1000 + n - 1, c.byref(ht), None) == ALK_OK
    status, hst = StageStatus(), HtStatus()
    pay = (c.c_int32 * 1)(1)
    try:
        rc = L.alk_pipeline_build_async(cols, 2, 1, mode, c.byref(prog), None, -1, ht, 0, pay, 0, c.byref(status),
                                        None)
        assert rc == ALK_OK
        assert L.alk_ht_info_async(ht, c.byref(hst), None) == ALK_OK
        torch.cuda.synchronize()
        assert status.err == ALK_OK and status.rows_in == n and status.hits == int(sel.sum())
        assert hst.inserted == int(sel.sum()) and list(hst.flags) == [0, 0, 0, 0]
        # keys and payload by table position (gathered with the identity permutation):
        # every inserted key carries its own row's value
        slots = L.alk_ht_slots(ht)
        got = torch.empty(2 * slots, dtype=torch.int64, device="cuda")
        ident = torch.arange(slots, dtype=torch.int32, device="cuda")
        cnt = torch.tensor([slots], dtype=torch.int64, device="cuda")
        colp = (c.c_void_p * 2)(L.alk_ht_keys(ht), L.alk_ht_payload(ht, 0))
        assert L.alk_gather_rows(colp, 2, ident.data_ptr(), cnt.data_ptr(), slots, got.data_ptr(), None) == ALK_OK
        torch.cuda.synchronize()
        tk, tv = got.cpu().numpy()[:slots], got.cpu().numpy()[slots:]
        occ = tk != np.int64(np.uint64(0x8080808080808080).view(np.int64))
        assert dict(zip(tk[occ].tolist(), tv[occ].tolist())) == dict(zip(keys[sel].tolist(), vals[sel].tolist()))
    finally:
        L.alk_ht_free(ht, None)
        torch.cuda.synchronize()
    del kb, vb


@pytest.mark.parametrize("route", ["records", "positions"])
@pytest.mark.parametrize("dup", [False, True])
def test_dense_build(route, dup):
    """Dense (rank-addressed) table: slots are the keys' ranks, so the key column comes out
    sorted and each key carries its row's payload. 'records': no predicate, so the
    TMA-staged scan records [position, key, payload] itself; 'positions': a predicate that
    is not a conjunction runs the register-machine scan, then the bitmap pass. A repeated
    key is reported as a duplicate on either route."""
    import torch
    L = _lib()
    L.alk_ht_create_dense.argtypes = [c.c_uint64, c.c_uint32, c.c_int64, c.c_int64, c.POINTER(c.c_void_p),
                                      c.c_void_p]
    rng = np.random.default_rng(11)
    n = 300_000
    keys = rng.permutation(n).astype(np.int64) * 3 + 11
    if dup:
        keys[-1] = keys[0]
    vals = rng.integers(0, 1 << 30, n).astype(np.int64)
    kb, ks = _column(keys)
    vb, vs = _column(vals)
    cols = (ColSeg * 2)(ks, vs)
    mode = (c.c_uint8 * 1)(2)
    pred = _or_pred(1, 0) if route == "positions" else None
    ht = c.c_void_p()
    assert L.alk_ht_create_dense(n + 16, 1, int(keys.min()), int(keys.max()), c.byref(ht), None) == ALK_OK
    pay = (c.c_int32 * 1)(1)
    try:
        rows_in, hits = c.c_uint64(), c.c_uint64()
        rc = L.alk_pipeline_build(cols, 2, 1, mode, c.byref(pred) if pred else None, None, -1, ht, 0, pay, 0,
                                  c.byref(rows_in), c.byref(hits), None)
        assert rc == ALK_OK and rows_in.value == n
        ins, fl = c.c_uint64(), c.c_int()
        assert L.alk_ht_info(ht, c.byref(ins), c.byref(fl), None) == ALK_OK
        distinct = np.unique(keys)
        assert ins.value == len(distinct)
        assert (fl.value & 1) == (1 if dup else 0)
        if dup:
            return
        got = torch.empty(2 * n, dtype=torch.int64, device="cuda")
        ident = torch.arange(n, dtype=torch.int32, device="cuda")
        cnt = torch.tensor([n], dtype=torch.int64, device="cuda")
        colp = (c.c_void_p * 2)(L.alk_ht_keys(ht), L.alk_ht_payload(ht, 0))
        assert L.alk_gather_rows(colp, 2, ident.data_ptr(), cnt.data_ptr(), n, got.data_ptr(), None) == ALK_OK
        torch.cuda.synchronize()
        tk, tv = got.cpu().numpy()[:n], got.cpu().numpy()[n:]
        order = np.argsort(keys)
        assert np.array_equal(tk, keys[order])  # slot = rank of the key
        assert np.array_equal(tv, vals[order])
    finally:
        L.alk_ht_free(ht, None)
        torch.cuda.synchronize()
    del kb, vb


@pytest.mark.parametrize("k", [1, 10, 16])
def test_topk_select_and_gather_rows(k):
    import torch
    L = _lib()
    rng = np.random.default_rng(k)
    n = 1_000_003
    rank = rng.integers(-5000, 5000, n).astype(np.int64)  # many ties
    live = (rng.random(n) < 0.3).astype(np.uint64) * rng.integers(1, 9, n).astype(np.uint64)
    other = rng.integers(0, 1 << 40, n).astype(np.int64)
    d_rank = torch.from_numpy(rank).cuda()
    d_live = torch.from_numpy(live.view(np.int64)).cuda()
    d_other = torch.from_numpy(other).cuda()
    cap = 1 << 16
    d_out = torch.zeros(cap, dtype=torch.int32, device="cuda")
    d_cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    assert L.alk_topk_select(d_rank.data_ptr(), d_live.data_ptr(), n, k, d_out.data_ptr(), cap, d_cnt.data_ptr(),
                             None) == ALK_OK
    small = 4096
    d_rows = torch.zeros(2 * small, dtype=torch.int64, device="cuda")
    cols = (c.c_void_p * 2)(d_rank.data_ptr(), d_other.data_ptr())
    assert L.alk_gather_rows(cols, 2, d_out.data_ptr(), d_cnt.data_ptr(), small, d_rows.data_ptr(), None) == ALK_OK
    torch.cuda.synchronize()
    m = int(d_cnt.item())
    lv = rank[live != 0]
    thr = np.sort(lv)[::-1][k - 1]
    want = np.nonzero((live != 0) & (rank >= thr))[0]
    assert m == len(want)
    got = np.sort(d_out.cpu().numpy()[:m].astype(np.int64))
    assert np.array_equal(got, want)
    rows = d_rows.cpu().numpy()
    idx = d_out.cpu().numpy()[:min(m, small)].astype(np.int64)
    assert np.array_equal(rows[:len(idx)], rank[idx])
    assert np.array_equal(rows[small:small + len(idx)], other[idx])


ALK_ERR_ARG, ALK_DENSE_FULL, ALK_DENSE_RANKS, ALK_DENSE_BITS = 1, 0, 1, 2


def _lt_pred(slot, c0, conjunctive):
    """column(slot) < c0; as a single conjunct, or (not a conjunction) OR-ed with
    column(slot) < -1, which no row meets."""
    p = Program()
    p.consts[0] = c0
    p.ins[0] = Instr(ALK_OP_LT, 0, ALK_K_COL, ALK_K_CONST, slot, 0, 0)
    if conjunctive:
        p.n_instr, p.result = 1, 0
        return p
    p.consts[1] = -1
    p.n_instr, p.result = 3, 2
    p.ins[1] = Instr(ALK_OP_LT, 1, ALK_K_COL, ALK_K_CONST, slot, 1, 0)
    p.ins[2] = Instr(ALK_OP_OR, 2, ALK_K_REG, ALK_K_REG, 0, 1, 0)
    return p


@pytest.mark.parametrize("route", ["blocked", "positions"])
@pytest.mark.parametrize("dup", [None, "filtered", "skipped"])
def test_dense_modes_and_late_rows(route, dup):
    """Ranks-only and membership-only dense tables, and the late fetch of keys and
    payload for candidate slots. Three segments of ascending, disjoint key ranges, the
    middle one skipped; a predicate keeps 60% of the rows. 'blocked': a one-conjunct
    predicate on narrow columns runs the blocked scan, which sets the bits itself;
    'positions': a predicate that is not a conjunction goes through the survivor list and
    the bitmap pass. dup 'filtered': a row the predicate removes repeats a candidate's key,
    so the late fetch cannot tell the rows apart and reports it; 'skipped': the repeat
    sits in the skipped segment, which the fetch does not read. alk_seg_sorted tells the
    ascending segments from a shuffled one."""
    import torch
    L = _lib()
    vp, u32, u64, i32, i64 = c.c_void_p, c.c_uint32, c.c_uint64, c.c_int32, c.c_int64
    L.alk_ht_create_dense_mode.argtypes = [u64, u32, i64, i64, c.c_int, c.POINTER(vp), vp]
    L.alk_ht_late_rows.argtypes = [vp, vp, vp, u32, c.POINTER(ColSeg), u32, u32, c.POINTER(c.c_uint8),
                                   c.POINTER(i64), c.POINTER(i64), c.POINTER(vp), vp, vp]
    L.alk_seg_sorted.argtypes = [c.POINTER(ColSeg), u32, c.POINTER(c.c_uint8), vp]
    rng = np.random.default_rng(21)
    per, nseg = 100_000, 3
    keys = np.arange(per * nseg, dtype=np.int64) * 3 + 11
    filt = rng.integers(0, 100, per * nseg).astype(np.int64)
    pay0 = rng.integers(-(1 << 20), 1 << 20, per * nseg).astype(np.int64)
    pay1 = rng.integers(-(1 << 50), 1 << 50, per * nseg).astype(np.int64)
    seg_mode = [2, 0, 2]
    live = (filt < 60) & np.repeat(np.array(seg_mode) != 0, per)
    dup_key = None
    if dup == "filtered":  # the next row, filtered out, repeats a survivor's key (order kept)
        src = int(np.nonzero(live[:per - 1] & ~live[1:per])[0][5])
        dup_key = int(keys[src])
        keys[src + 1] = dup_key
    elif dup == "skipped":  # the skipped segment's first row repeats a survivor's key
        src = int(np.nonzero(live[:per])[0][-3])
        dup_key = int(keys[src])
        keys[per] = dup_key
    bufs, segs = [], []
    for col, bits in ((keys, 32), (filt, 8), (pay0, 32), (pay1, 64)):
        for g in range(nseg):
            b, cs = _column(col[g * per:(g + 1) * per], bits)
            bufs.append(b)
            segs.append(cs)
    cols = (ColSeg * len(segs))(*segs)
    mode = (c.c_uint8 * nseg)(*seg_mode)
    asc = (c.c_uint8 * (nseg + 1))()
    b, shuffled = _column(rng.permutation(keys[:per]), 32)
    bufs.append(b)
    assert L.alk_seg_sorted((ColSeg * (nseg + 1))(*(segs[:nseg] + [shuffled])), nseg + 1, asc, None) == ALK_OK
    assert list(asc) == [1, 1, 1, 0]
    pred = _lt_pred(1, 60, route == "blocked")
    kmin, kmax = int(keys.min()), int(keys.max())
    skeys = np.sort(keys[live])
    want = {int(keys[r]): int(r) for r in np.nonzero(live)[0]}  # key -> its surviving row
    # membership only: counts and flags, no slots; payload and late fetch refused
    ht = c.c_void_p()
    assert L.alk_ht_create_dense_mode(len(keys), 1, kmin, kmax, ALK_DENSE_BITS, c.byref(ht), None) == ALK_ERR_ARG
    assert L.alk_ht_create_dense_mode(len(keys), 0, kmin, kmax, ALK_DENSE_BITS, c.byref(ht), None) == ALK_OK
    rows_in, hits = c.c_uint64(), c.c_uint64()
    ins, fl = c.c_uint64(), c.c_int()
    try:
        assert L.alk_pipeline_build(cols, 4, nseg, mode, c.byref(pred), None, -1, ht, 0, None, 0, c.byref(rows_in),
                                    c.byref(hits), None) == ALK_OK
        assert L.alk_ht_info(ht, c.byref(ins), c.byref(fl), None) == ALK_OK
        assert ins.value == len(skeys) and fl.value == 0
        assert not L.alk_ht_keys(ht) and not L.alk_ht_payload(ht, 0)
    finally:
        L.alk_ht_free(ht, None)
        torch.cuda.synchronize()
    # ranks only: slots are ranks; the late fetch names every candidate's key and row
    ht = c.c_void_p()
    assert L.alk_ht_create_dense_mode(len(keys), 0, kmin, kmax, ALK_DENSE_RANKS, c.byref(ht), None) == ALK_OK
    try:
        assert L.alk_pipeline_build(cols, 4, nseg, mode, c.byref(pred), None, -1, ht, 0, None, 0, c.byref(rows_in),
                                    c.byref(hits), None) == ALK_OK
        assert L.alk_ht_info(ht, c.byref(ins), c.byref(fl), None) == ALK_OK
        assert ins.value == len(skeys) and fl.value == 0
        slots = L.alk_ht_slots(ht)
        cand = rng.choice(len(skeys), 300, replace=False).astype(np.int64)
        cand[1] = 0  # the first and the last key
        cand[2] = len(skeys) - 1
        if dup_key is not None:
            cand[0] = int(np.searchsorted(skeys, dup_key))
        cand = np.unique(cand)
        d_cand = torch.from_numpy(cand.astype(np.int32)).cuda()
        d_cnt = torch.tensor([len(cand)], dtype=torch.int64, device="cuda")
        outs = [torch.full((slots,), -7, dtype=torch.int64, device="cuda") for _ in range(3)]
        outp = (c.c_void_p * 3)(*[o.data_ptr() for o in outs])
        st = torch.zeros(1, dtype=torch.int32, device="cuda")
        late_cols = (ColSeg * (3 * nseg))(*(segs[:nseg] + segs[2 * nseg:]))
        lo = (c.c_int64 * nseg)(*[int(keys[g * per:(g + 1) * per].min()) for g in range(nseg)])
        hi = (c.c_int64 * nseg)(*[int(keys[g * per:(g + 1) * per].max()) for g in range(nseg)])
        rc = L.alk_ht_late_rows(ht, d_cand.data_ptr(), d_cnt.data_ptr(), 1 << 16, late_cols, 2, nseg, mode, lo, hi,
                                outp, st.data_ptr(), None)
        assert rc == ALK_OK
        torch.cuda.synchronize()
        assert int(st.item()) == (1 if dup == "filtered" else 0)
        ok = cand
        if dup == "filtered":  # the ambiguous candidate aside
            ok = cand[skeys[cand] != dup_key]
        got = [o.cpu().numpy() for o in outs]
        assert np.array_equal(got[0][cand], skeys[cand])
        rows = np.array([want[int(k)] for k in skeys[ok]])
        assert np.array_equal(got[1][ok], pay0[rows])
        assert np.array_equal(got[2][ok], pay1[rows])
        untouched = np.setdiff1d(np.arange(slots), cand)
        assert (got[0][untouched] == -7).all()
    finally:
        L.alk_ht_free(ht, None)
        torch.cuda.synchronize()
    del bufs


@pytest.mark.parametrize("span,bits", [(0, 8), (255, 8), (256, 16), (65535, 16), (1 << 20, 32), ((1 << 32) - 1, 32),
                                       (1 << 40, 64)])
def test_for_reencode_picks_the_narrowest_width(span, bits):
    """alk_for_reencode (how FOR-delta segments stay resident): exact minimum, the
    narrowest width that holds the span, and the values less the minimum at that width;
    a too small output is refused."""
    import torch
    L = ab.lib()
    L.alk_for_reencode.argtypes = [c.c_void_p, c.c_uint64, c.c_void_p, c.c_size_t, c.POINTER(c.c_int64),
                                   c.POINTER(c.c_uint32), c.c_void_p]
    rng = np.random.default_rng(span % 1000 + 3)
    n = 100_003
    lo = -(1 << 35) + 17
    v = lo + rng.integers(0, span + 1, n, dtype=np.int64)
    v[0], v[-1] = lo, lo + span  # both ends present: the span is exact
    d_in = torch.from_numpy(v).cuda()
    out = torch.zeros(n * 8 // 8 + 32, dtype=torch.int64, device="cuda")
    low, b = c.c_int64(), c.c_uint32()
    # one byte short of the width it needs: refused
    assert L.alk_for_reencode(d_in.data_ptr(), n, out.data_ptr(), n * bits // 8 - 1, c.byref(low), c.byref(b),
                              None) == ALK_ERR_OVERFLOW
    assert L.alk_for_reencode(d_in.data_ptr(), n, out.data_ptr(), n * 8, c.byref(low), c.byref(b), None) == ALK_OK
    torch.cuda.synchronize()
    assert low.value == lo and b.value == bits
    dt = {8: np.uint8, 16: np.uint16, 32: np.uint32, 64: np.uint64}[bits]
    got = out.cpu().numpy().view(np.uint8)[:n * bits // 8].view(dt).astype(np.uint64)
    assert np.array_equal(got, (v - lo).astype(np.uint64))
