"""The learned cardinality estimator on the device.

Kernels against the CPU oracle (oracle/mlp.py): the forward pass, the gradient of the
masked MSE for every parameter, and an Adam step, all with BF16 weights and FP32
accumulation (tolerances below are relative to each quantity's scale). The exact
per-segment counting pass and the histograms against numpy (bit-exact). Then the engine
loop: records of exact counts from fused three-way queries, training on the GPU, q-error
on held-out (query, segment) records against the classical estimate (histograms and
independence), and first runs sized by the estimator: the same STORE output, far fewer
bytes reserved than the upper-bound sizing used without it."""
import ctypes as c
import os
import sys

import numpy as np
import pytest

import alenka_b200 as ab
from alenka_b200 import workloads as wl

from . import _oracle
from .test_gpu_stages import ALK_K_COL, ALK_K_CONST, ALK_OP_LT, ColSeg, Instr, Program, _column, _lib

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import mlp  # noqa: E402

pytestmark = pytest.mark.gpu


def _ptr(t):
    return c.c_void_p(t.data_ptr())


class _Net:
    def __init__(self, seed):
        self.L = ab.lib()
        self.h = c.c_void_p()
        assert self.L.alk_mlp_create(seed, c.byref(self.h), None) == 0
        self.n = self.L.alk_mlp_param_count()

    def params(self):
        m = np.zeros(self.n, np.float32)
        b = np.zeros(self.n, np.uint16)
        assert self.L.alk_mlp_params(self.h, m.ctypes.data_as(c.POINTER(c.c_float)),
                                     b.ctypes.data_as(c.POINTER(c.c_uint16)), None) == 0
        return m, b

    def close(self):
        self.L.alk_mlp_free(self.h, None)


def _data(n, seed):
    import torch
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 1, (n, 64)).astype(np.float32)
    t = rng.normal(-2, 1, (n, 3)).astype(np.float32)
    m = (rng.random((n, 3)) < 0.8).astype(np.float32)
    return x, t, m, [torch.from_numpy(a).cuda() for a in (x, t, m)]


def test_param_layout_and_bf16_copies():
    net = _Net(7)
    try:
        assert net.n == mlp.N_PARAMS
        master, bits = net.params()
        # the BF16 copies are the round-to-nearest-even values of the master weights
        np.testing.assert_array_equal(mlp.bf16_bits_to_f32(bits), mlp.bf16_round(master))
        W1 = mlp.unpack(master)[0]
        assert 0.05 < np.abs(W1).max() <= np.sqrt(6 / 64) + 1e-6
    finally:
        net.close()


def test_forward_matches_oracle():
    import torch
    net = _Net(3)
    try:
        x, _, _, (dx, _, _) = _data(1000, 1)
        dy = torch.zeros((1000, 3), dtype=torch.float32, device="cuda")
        assert net.L.alk_mlp_forward(net.h, _ptr(dx), 1000, _ptr(dy), None) == 0
        torch.cuda.synchronize()
        master, _ = net.params()
        want, _ = mlp.forward(master, x)
        got = dy.cpu().numpy()
        # FP32 accumulation over 64/128 terms against float64: well inside 1e-4 of scale
        np.testing.assert_allclose(got, want, rtol=1e-4, atol=1e-4 * np.abs(want).max())
    finally:
        net.close()


@pytest.mark.parametrize("n", [1, 37, 512])
def test_gradients_match_oracle(n):
    import torch
    net = _Net(11)
    try:
        x, t, m, (dx, dt, dm) = _data(n, n)
        g = torch.zeros(net.n, dtype=torch.float32, device="cuda")
        loss = c.c_float()
        assert net.L.alk_mlp_gradients(net.h, _ptr(dx), _ptr(dt), _ptr(dm), n, _ptr(g), c.byref(loss), None) == 0
        master, _ = net.params()
        want_loss, want = mlp.loss_and_grad(master, x, t, m)
        got = g.cpu().numpy()
        assert abs(loss.value - want_loss) <= 1e-4 * max(1.0, want_loss)
        # per parameter block, relative to the block's largest gradient
        o = 0
        for shape in mlp.SHAPES:
            k = int(np.prod(shape))
            scale = max(np.abs(want[o:o + k]).max(), 1e-12)
            np.testing.assert_allclose(got[o:o + k], want[o:o + k], rtol=0, atol=2e-4 * scale)
            o += k
        # the direction agrees to within rounding
        cos = got @ want / (np.linalg.norm(got) * np.linalg.norm(want))
        assert cos > 0.99999
    finally:
        net.close()


def test_adam_step_matches_oracle():
    import torch
    net = _Net(5)
    try:
        n = 256
        x, t, m, (dx, dt, dm) = _data(n, 9)
        p0, _ = net.params()
        _, g = mlp.loss_and_grad(p0, x, t, m)
        lr = 1e-3
        want, _, _ = mlp.adam_step(p0.astype(np.float64), g, np.zeros_like(g), np.zeros_like(g), 1, lr)
        loss = c.c_float()
        # one epoch of one batch is one Adam step
        assert net.L.alk_mlp_train(net.h, _ptr(dx), _ptr(dt), _ptr(dm), n, 1, n, lr, c.byref(loss), None) == 0
        p1, _ = net.params()
        # the first step moves every parameter with a non-negligible gradient by ~lr
        big = np.abs(g) > 1e-3 * np.abs(g).max()
        np.testing.assert_allclose(p1[big], want[big], rtol=0, atol=2e-6)
    finally:
        net.close()


def test_training_reduces_loss():
    net = _Net(2)
    try:
        import torch
        rng = np.random.default_rng(4)
        x = rng.random((4096, 64)).astype(np.float32)
        w = rng.normal(0, 1, (64, 3)).astype(np.float32)
        t = np.tanh(x @ w / 8).astype(np.float32)  # a smooth target the network can fit
        m = np.ones_like(t)
        dx, dt, dm = (torch.from_numpy(a).cuda() for a in (x, t, m))
        l0, l1 = c.c_float(), c.c_float()
        assert net.L.alk_mlp_train(net.h, _ptr(dx), _ptr(dt), _ptr(dm), 4096, 1, 128, 1e-3, c.byref(l0), None) == 0
        assert net.L.alk_mlp_train(net.h, _ptr(dx), _ptr(dt), _ptr(dm), 4096, 40, 128, 1e-3, c.byref(l1), None) == 0
        assert l1.value < 0.1 * l0.value
    finally:
        net.close()


def test_hist16_and_exact_counts_match_numpy():
    import torch
    L = _lib()
    rng = np.random.default_rng(8)
    segs = [rng.integers(1000, 9000, 70_001), rng.integers(5000, 5600, 33_333), rng.integers(0, 100, 1)]
    keys = [rng.integers(0, 50_000, len(v)) for v in segs]
    bufs, cs_v, cs_k = [], [], []
    for v, k in zip(segs, keys):
        b1, c1 = _column(v.astype(np.int64))
        b2, c2 = _column(k.astype(np.int64))
        bufs += [b1, b2]
        cs_v.append(c1)
        cs_k.append(c2)
    nseg = len(segs)
    cols = (ColSeg * (2 * nseg))(*cs_v, *cs_k)
    # histograms over each segment's [min, max]
    h = torch.zeros(16, dtype=torch.int32, device="cuda")
    for g, v in enumerate(segs):
        lo, hi = int(v.min()), int(v.max())
        assert L.alk_card_hist16(c.byref(cols[g]), lo, hi, _ptr(h), None) == 0
        torch.cuda.synchronize()
        span = hi - lo + 1
        b = np.minimum(((v - lo) / span * 16).astype(np.int64), 15)
        np.testing.assert_array_equal(h.cpu().numpy(), np.bincount(b, minlength=16))
    # value < 5300, probing a table of the even keys below 40000, distinct probe keys
    p = Program()
    p.n_instr, p.result = 1, 0
    p.consts[0] = 5300
    p.ins[0] = Instr(ALK_OP_LT, 0, ALK_K_COL, ALK_K_CONST, 0, 0, 0)
    build = np.arange(0, 40_000, 2, dtype=np.int64)
    ht = c.c_void_p()
    assert L.alk_ht_create_range(len(build), 0, 0, 49_999, c.byref(ht), None) == 0
    try:
        bb, bc = _column(build)
        bcols = (ColSeg * 1)(bc)
        mode1 = (c.c_uint8 * 1)(1)
        rows_in, hits = c.c_uint64(), c.c_uint64()
        assert L.alk_pipeline_build(bcols, 1, 1, mode1, None, None, -1, ht, 0, None, 0, c.byref(rows_in),
                                    c.byref(hits), None) == 0
        mode = (c.c_uint8 * nseg)(2, 2, 0)
        out = (c.c_uint64 * (3 * nseg))()
        assert L.alk_card_count(cols, 2, nseg, mode, c.byref(p), ht, 1, 1, 0, 49_999, out, None) == 0
        for g, (v, k) in enumerate(zip(segs, keys)):
            if mode[g] == 0:
                assert list(out[3 * g:3 * g + 3]) == [0, 0, 0]
                continue
            f = v < 5300
            j = f & (k < 40_000) & (k % 2 == 0)
            assert out[3 * g] == f.sum()
            assert out[3 * g + 1] == j.sum()
            assert out[3 * g + 2] == len(np.unique(k[j]))
        # without a key column the distinct count is unknown
        assert L.alk_card_count(cols, 2, nseg, mode, c.byref(p), None, -1, -1, 0, -1, out, None) == 0
        assert out[0] == (segs[0] < 5300).sum() and out[1] == out[0] and out[2] == 2 ** 64 - 1
    finally:
        L.alk_ht_free(ht, None)


# ------------------------------------------------------------------ engine loop


@pytest.fixture(scope="module")
def card_tables(tmp_path_factory):
    d = tmp_path_factory.mktemp("card")
    wl.make_three_way(str(d), scale=0.02, seg_rows=50_000, seed=21)
    return str(d)


def _run(s, script):
    try:
        s.execute(script)
    except ab.AlenkaError as e:  # an empty join: the reference's error, recorded all the same
        return "error: " + str(e)
    return None


def _qerr(pred, act):
    return np.exp(np.abs(pred - act))


def test_estimator_records_train_and_size_first_runs(card_tables):
    d = card_tables
    # about 100k (query, segment) records: 3000 training queries of ~31 segments each
    n_train, n_test = 3000, 200
    with ab.Session(d) as s:
        s.card_mode(record=True)
        bounds = [0]
        for q in range(n_train + n_test):
            _run(s, wl.card_script(q, out="qc.txt"))
            if q + 1 == n_train:
                bounds.append(len(s.card_records()[1]))
        x, y, m = s.card_records()
        bounds.append(len(y))
        assert len(y) == bounds[-1] and len(y) >= 25 * (n_train + n_test)
        split = bounds[1]
        l_first = s.card_train(0, split, epochs=1, batch=256, lr=1e-3, seed=3)
        l_last = s.card_train(0, split, epochs=60, batch=256, lr=1e-3, seed=4)
        assert l_last < 0.25 * l_first
        # held-out (query, segment) records: q-error of the rows passing filter and probe
        xt, yt, mt = x[split:], y[split:], m[split:]
        pt = np.minimum(s.card_predict(xt), 0.0)
        rows = np.exp2(xt[:, 3] * 32) - 1
        floor = np.log(0.5 / np.maximum(rows, 1))
        act = yt[:, 0] + yt[:, 1] * mt[:, 1]
        est = pt[:, 0] + pt[:, 1] * mt[:, 1]
        classical = np.maximum(np.log(np.maximum(xt[:, 9] * np.where(mt[:, 1] > 0, xt[:, 10], 1.0), 1e-30)), floor)
        q_mlp, q_cls = _qerr(est, act), _qerr(classical, act)
        med_mlp, med_cls = np.median(q_mlp), np.median(q_cls)
        p95_mlp, p95_cls = np.percentile(q_mlp, 95), np.percentile(q_cls, 95)
        print(f"\nq-error (filter x probe, {len(act)} held-out records): "
              f"MLP median {med_mlp:.3f} p95 {p95_mlp:.3f}; classical median {med_cls:.3f} p95 {p95_cls:.3f}")
        assert med_mlp < med_cls and p95_mlp < p95_cls
        assert med_mlp < 1.3 and p95_mlp < 10

        # first runs of new queries: without the estimator (upper-bound sizing), then with it
        s.card_mode(record=False, use=False)
        outs, reserved = {}, {}
        for use in (False, True):
            s.card_mode(record=False, use=use)
            res, tot, reruns = [], 0, 0
            for q in range(1000, 1012):
                s.card_forget()
                err = _run(s, wl.card_script(q, out="qc.txt"))
                st = s.stats()
                tot += st.reserved_bytes
                reruns += st.card_reruns
                if use and err is None:
                    assert st.card_estimates >= 3
                with open(os.path.join(d, "qc.txt"), "rb") as f:
                    res.append(err or f.read())
            outs[use], reserved[use] = res, tot
            print(f"use={use}: reserved {tot / 2**20:.1f} MiB over 12 first runs, reruns {reruns}")
        assert outs[True] == outs[False]
        assert reserved[True] < 0.5 * reserved[False]


def test_record_mode_keeps_results_exact(card_tables):
    d = card_tables
    for q in (3, 4):
        script = wl.card_script(q, out="qr.txt")
        try:
            _oracle.execute(d, script.replace("qr.txt", "oracle_qr.txt"))
            want = open(os.path.join(d, "oracle_qr.txt"), "rb").read()
        except RuntimeError as e:
            want = None
        with ab.Session(d) as s:
            s.card_mode(record=True)
            if want is None:
                with pytest.raises(ab.AlenkaError):
                    s.execute(script)
                continue
            s.execute(script)
            assert s.stats().plan == 1
        assert open(os.path.join(d, "qr.txt"), "rb").read() == want


def test_estimator_save_and_load(card_tables, tmp_path):
    d = card_tables
    with ab.Session(d) as s:
        s.card_mode(record=True)
        for q in range(40):
            _run(s, wl.card_script(5000 + q, out="qs.txt"))
        x, _, _ = s.card_records()
        s.card_train(0, len(x), epochs=3, batch=128, lr=1e-3, seed=9)
        want = s.card_predict(x[:500])
        f = tmp_path / "card.bin"
        s.card_save(f)
    with ab.Session(d) as s2:
        with pytest.raises(ab.AlenkaError):
            s2.card_predict(x[:10])  # nothing trained or loaded yet
        s2.card_load(f)
        np.testing.assert_array_equal(s2.card_predict(x[:500]), want)
        bad = tmp_path / "bad.bin"
        bad.write_bytes(b"not a network")
        with pytest.raises(ab.AlenkaError):
            s2.card_load(bad)
