"""alenka_b200: a B200 (sm_100a) engine for Alenka's columnar scan -> filter -> join ->
group-by -> order path, behind the reference's own embedding API (alenkaInit /
alenkaExecute / alenkaClose) and operator entry points.

This module is a thin ctypes binding of the in-tree ``libalenka_b200.so``; there is no
Python or CPU execution path. Importing it on a machine without the built library raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libalenka_b200.so")

ALK_OK = 0
ALK_ERR_OVERFLOW = 3
ALK_ERR_UNSUPPORTED = 5
ALK_SESSION_RESIDENT = 1
ALK_SESSION_PLAIN = 2
ALK_SESSION_NOGRAPH = 4
ALK_SESSION_DELTA = 8

_lib = None


class AlenkaError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"status {code}: {msg}")
        self.code = code


class Stats(ctypes.Structure):
    _fields_ = [
        ("rows_scanned", ctypes.c_uint64),
        ("kernels", ctypes.c_uint64),
        ("h2d_bytes", ctypes.c_uint64),
        ("d2h_bytes", ctypes.c_uint64),
        ("plan", ctypes.c_uint32),
        ("segments_skipped", ctypes.c_uint32),
        ("hot_kernel_ms", ctypes.c_double),
        ("hot_kernel_bytes", ctypes.c_uint64),
        ("hot_kernel_launches", ctypes.c_uint64),
        ("query_device_ms", ctypes.c_double),
        ("reserved_bytes", ctypes.c_uint64),
        ("card_estimates", ctypes.c_uint32),
        ("card_reruns", ctypes.c_uint32),
        ("batch_host_ms", ctypes.c_double * 3),
        ("sort_groupbys", ctypes.c_uint32),
        ("hash_groupbys", ctypes.c_uint32),
    ]


class Tuning(ctypes.Structure):
    _fields_ = [("consumer_warps", ctypes.c_uint32), ("stages", ctypes.c_uint32), ("blocks_per_sm", ctypes.c_uint32)]


def _declare(L):
    c = ctypes
    vp, u32, u64, i64, i32 = c.c_void_p, c.c_uint32, c.c_uint64, c.c_int64, c.c_int
    L.alk_session_open.argtypes = [c.c_char_p, u32, c.POINTER(vp)]
    L.alk_session_execute.argtypes = [vp, c.c_char_p]
    L.alk_session_error.argtypes = [vp]
    L.alk_session_error.restype = c.c_char_p
    L.alk_session_stream.argtypes = [vp]
    L.alk_session_stream.restype = vp
    L.alk_session_preload.argtypes = [vp, c.c_char_p]
    L.alk_session_stats.argtypes = [vp, c.POINTER(Stats)]
    L.alk_session_set_timing.argtypes = [vp, i32]
    L.alk_session_close.argtypes = [vp]
    L.alk_session_close.restype = None
    L.alk_gen_lineitem_flat.argtypes = [c.c_char_p, u64, u32, u64, i32, c.c_char_p, i32]
    L.alk_gen_names.argtypes = [c.c_char_p, u64, u32, u32, u64, c.c_char_p, i32]
    L.alk_gen_three_way.argtypes = [c.c_char_p, u64, u64, u64, u32, u64, i32, c.c_char_p, i32]
    L.alk_gen_three_way_zipf.argtypes = [c.c_char_p, u64, u64, u64, u32, u64, i32, c.c_double, c.c_char_p, i32]
    L.alk_date_add_days.argtypes = [i64, i64]
    L.alk_date_add_days.restype = i64
    L.alk_decode_segment.argtypes = [vp, u32, u32, u32, i64, i64, u32, vp, vp]
    L.alk_hash_tuples.argtypes = [c.POINTER(vp), u32, u64, u32, vp, vp]
    L.alk_groupby_hash.argtypes = [c.POINTER(vp), u32, c.POINTER(vp), c.POINTER(c.c_uint8), u32, u64,
                                   c.POINTER(vp), c.POINTER(vp), vp, c.POINTER(u64), vp]
    L.alk_sort_perm.argtypes = [c.POINTER(vp), c.POINTER(c.c_uint8), u32, u64, vp, vp]
    L.alk_sort_perm_u64.argtypes = [vp, u64, vp, vp]
    L.alk_gather.argtypes = [vp, vp, u64, vp, vp]
    L.alk_join_build.argtypes = [vp, u64, c.POINTER(vp), vp]
    L.alk_join_probe.argtypes = [vp, vp, u64, vp, vp, u64, c.POINTER(u64), vp]
    L.alk_join_free.argtypes = [vp, vp]
    L.alk_join_free.restype = None
    L.alk_device_info.argtypes = [c.POINTER(i32), c.POINTER(i32), c.POINTER(i32)]
    fp = c.POINTER(c.c_float)
    L.alk_mlp_param_count.restype = u32
    L.alk_mlp_create.argtypes = [u64, c.POINTER(vp), vp]
    L.alk_mlp_free.argtypes = [vp, vp]
    L.alk_mlp_free.restype = None
    L.alk_mlp_set_params.argtypes = [vp, fp, vp]
    L.alk_mlp_params.argtypes = [vp, fp, c.POINTER(c.c_uint16), vp]
    L.alk_mlp_forward.argtypes = [vp, vp, u64, vp, vp]
    L.alk_mlp_gradients.argtypes = [vp, vp, vp, vp, u64, vp, fp, vp]
    L.alk_mlp_train.argtypes = [vp, vp, vp, vp, u64, u32, u32, c.c_float, fp, vp]
    L.alk_card_hist16.argtypes = [vp, i64, i64, vp, vp]
    L.alk_card_count.argtypes = [vp, u32, u32, vp, vp, vp, i32, i32, i64, i64, c.POINTER(u64), vp]
    L.alk_session_execute_batch.argtypes = [vp, c.POINTER(c.c_char_p), u32]
    L.alk_session_tuning.argtypes = [vp, c.POINTER(Tuning), i32]
    L.alk_session_set_tuning.argtypes = [vp, c.POINTER(Tuning)]
    L.alk_session_set_plain.argtypes = [vp, i32]
    L.alk_session_set_groupby.argtypes = [vp, i32]
    L.alk_session_gen_flat_resident.argtypes = [vp, c.c_char_p, c.POINTER(u32), u32, u64, u64]
    L.alk_gen_flat_value.argtypes = [u64, i32, u64]
    L.alk_gen_flat_value.restype = i64
    L.alk_session_card_mode.argtypes = [vp, i32, i32]
    L.alk_session_card_records.argtypes = [vp, fp, fp, fp, u64, c.POINTER(u64)]
    L.alk_session_card_train.argtypes = [vp, u64, u64, u32, u32, c.c_float, u64, fp]
    L.alk_session_card_predict.argtypes = [vp, fp, u64, fp]
    L.alk_session_card_forget.argtypes = [vp]
    L.alk_session_card_save.argtypes = [vp, c.c_char_p]
    L.alk_session_card_load.argtypes = [vp, c.c_char_p]
    L.alenkaInit.argtypes = [c.POINTER(c.c_char_p)]
    L.alenkaInit.restype = None
    L.alenkaExecute.argtypes = [c.c_char_p]
    L.alenkaClose.argtypes = []
    L.alenkaClose.restype = None


def lib():
    """The loaded engine library (raises when it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing; build it with python -m alenka_b200.build")
        L = ctypes.CDLL(LIB_PATH)
        _declare(L)
        _lib = L
    return _lib


class Session:
    """An engine session over a data directory (data.dictionary + segment files)."""

    def __init__(self, data_dir, resident=True, plain=False, graphs=True, delta=False):
        flags = ((ALK_SESSION_RESIDENT if resident else 0) | (ALK_SESSION_PLAIN if plain else 0)
                 | (0 if graphs else ALK_SESSION_NOGRAPH) | (ALK_SESSION_DELTA if delta else 0))
        h = ctypes.c_void_p()
        rc = lib().alk_session_open(str(data_dir).encode(), flags, ctypes.byref(h))
        if rc != ALK_OK:
            raise AlenkaError(rc, "cannot open a session")
        self._h = h

    def execute(self, script):
        rc = lib().alk_session_execute(self._h, script.encode())
        if rc != ALK_OK:
            raise AlenkaError(rc, lib().alk_session_error(self._h).decode())

    def preload(self, table):
        rc = lib().alk_session_preload(self._h, table.encode())
        if rc != ALK_OK:
            raise AlenkaError(rc, lib().alk_session_error(self._h).decode())

    def stats(self):
        s = Stats()
        lib().alk_session_stats(self._h, ctypes.byref(s))
        return s

    def set_timing(self, on):
        lib().alk_session_set_timing(self._h, 1 if on else 0)

    def execute_batch(self, scripts):
        """Runs the scripts with one batched launch for their dense group-bys."""
        arr = (ctypes.c_char_p * len(scripts))(*[x.encode() for x in scripts])
        rc = lib().alk_session_execute_batch(self._h, arr, len(scripts))
        if rc != ALK_OK:
            raise AlenkaError(rc, lib().alk_session_error(self._h).decode())

    def gen_flat_resident(self, table, seg_rows, seed, row_base=0):
        """Generate a lineitem-shaped table in device memory (segments of seg_rows rows)."""
        arr = (ctypes.c_uint32 * len(seg_rows))(*seg_rows)
        rc = lib().alk_session_gen_flat_resident(self._h, table.encode(), arr, len(seg_rows), seed, row_base)
        if rc != ALK_OK:
            raise AlenkaError(rc, lib().alk_session_error(self._h).decode())

    def set_groupby(self, mode):
        """0: hash or sort by the expected group count; 1: hash; 2: sort."""
        if lib().alk_session_set_groupby(self._h, int(mode)) != ALK_OK:
            raise AlenkaError(1, "bad group-by mode")

    def set_plain(self, on):
        lib().alk_session_set_plain(self._h, 1 if on else 0)

    def tuning(self, autotune=None):
        """Launch shape of the last batched group-by; autotune True/False switches the
        autotuner."""
        t = Tuning()
        lib().alk_session_tuning(self._h, ctypes.byref(t), -1 if autotune is None else int(bool(autotune)))
        return (t.consumer_warps, t.stages, t.blocks_per_sm)

    def set_tuning(self, shape=None):
        """Fixes the batched group-by's launch shape (consumer_warps, stages,
        blocks_per_sm); None returns to the autotuner."""
        t = Tuning(*shape) if shape else None
        rc = lib().alk_session_set_tuning(self._h, ctypes.byref(t) if t else None)
        if rc:
            raise AlenkaError(rc, "bad launch shape %r" % (shape,))

    # ---- learned cardinality estimator
    def card_mode(self, record=False, use=False):
        lib().alk_session_card_mode(self._h, 1 if record else 0, 1 if use else 0)

    def card_records(self):
        """(features [n, 64], log-fraction targets [n, 3], target masks [n, 3]) as numpy."""
        import numpy as np
        n = ctypes.c_uint64()
        lib().alk_session_card_records(self._h, None, None, None, 0, ctypes.byref(n))
        x = np.zeros((n.value, 64), np.float32)
        y = np.zeros((n.value, 3), np.float32)
        m = np.zeros((n.value, 3), np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        lib().alk_session_card_records(self._h, x.ctypes.data_as(fp), y.ctypes.data_as(fp), m.ctypes.data_as(fp),
                                       n.value, ctypes.byref(n))
        return x, y, m

    def card_train(self, first, count, epochs=30, batch=256, lr=1e-3, seed=1):
        loss = ctypes.c_float()
        rc = lib().alk_session_card_train(self._h, first, count, epochs, batch, lr, seed, ctypes.byref(loss))
        if rc != ALK_OK:
            raise AlenkaError(rc, lib().alk_session_error(self._h).decode())
        return loss.value

    def card_predict(self, x):
        import numpy as np
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.zeros((x.shape[0], 3), np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        rc = lib().alk_session_card_predict(self._h, x.ctypes.data_as(fp), x.shape[0], y.ctypes.data_as(fp))
        if rc != ALK_OK:
            raise AlenkaError(rc, "estimator prediction failed")
        return y

    def card_save(self, path):
        rc = lib().alk_session_card_save(self._h, str(path).encode())
        if rc != ALK_OK:
            raise AlenkaError(rc, lib().alk_session_error(self._h).decode())

    def card_load(self, path):
        rc = lib().alk_session_card_load(self._h, str(path).encode())
        if rc != ALK_OK:
            raise AlenkaError(rc, lib().alk_session_error(self._h).decode())

    def card_forget(self):
        lib().alk_session_card_forget(self._h)

    @property
    def stream(self):
        return lib().alk_session_stream(self._h)

    def close(self):
        if self._h:
            lib().alk_session_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def gen_lineitem_flat(data_dir, rows, seg_rows, seed, delta=False):
    err = ctypes.create_string_buffer(512)
    rc = lib().alk_gen_lineitem_flat(str(data_dir).encode(), rows, seg_rows, seed, int(delta), err, 512)
    if rc:
        raise AlenkaError(rc, err.value.decode())


def gen_names(data_dir, rows, distinct, seg_rows, seed):
    err = ctypes.create_string_buffer(512)
    rc = lib().alk_gen_names(str(data_dir).encode(), rows, distinct, seg_rows, seed, err, 512)
    if rc:
        raise AlenkaError(rc, err.value.decode())


def gen_three_way(data_dir, customers, orders, lineitems, seg_rows, seed, delta=False, zipf=0.0):
    """Three-way tables; zipf > 0 draws lineitem's orderkeys from Zipf(zipf) over the
    orders (in key order)."""
    err = ctypes.create_string_buffer(512)
    if zipf > 0:
        rc = lib().alk_gen_three_way_zipf(str(data_dir).encode(), customers, orders, lineitems, seg_rows, seed,
                                          int(delta), float(zipf), err, 512)
    else:
        rc = lib().alk_gen_three_way(str(data_dir).encode(), customers, orders, lineitems, seg_rows, seed,
                                     int(delta), err, 512)
    if rc:
        raise AlenkaError(rc, err.value.decode())


def date_add_days(yyyymmdd, days):
    return lib().alk_date_add_days(yyyymmdd, days)
