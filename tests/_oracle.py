"""ctypes binding of the oracle (CPU restatement of the reference operators).
Test infrastructure only."""
import ctypes
import os

_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_lib = None


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(os.path.join(_ROOT, "oracle", "liboracle.so"))
        L.oracle_execute.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
        L.oracle_decode_segment.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t]
        L.oracle_decode_segment.restype = ctypes.c_int64
        L.oracle_murmur64a.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32]
        L.oracle_murmur64a.restype = ctypes.c_uint64
        L.oracle_rows_scanned.restype = ctypes.c_uint64
        _lib = L
    return _lib


def execute(data_dir, script, threads=0):
    err = ctypes.create_string_buffer(1024)
    rc = lib().oracle_execute(str(data_dir).encode(), script.encode(), threads, err, 1024)
    if rc:
        raise RuntimeError("oracle: " + err.value.decode())
    return lib().oracle_rows_scanned()


def decode_file(path):
    import numpy as np
    raw = open(path, "rb").read()
    buf = ctypes.create_string_buffer(raw, len(raw))
    rows = int.from_bytes(raw[len(raw) - 32 + 4:len(raw) - 32 + 8], "little")
    out = np.zeros(max(rows, 1), dtype=np.int64)
    n = lib().oracle_decode_segment(buf, len(raw), out.ctypes.data, out.size)
    if n < 0:
        raise ValueError("bad segment " + path)
    return out[:n]


def murmur64a(data: bytes, seed=100):
    buf = ctypes.create_string_buffer(data, len(data))
    return lib().oracle_murmur64a(buf, len(data), seed)
