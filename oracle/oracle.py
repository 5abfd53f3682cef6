"""TEST INFRASTRUCTURE ONLY — ctypes binding of the parity oracle.

The oracle is a CPU restatement of the reference's HTJ2K decoder
(frames-sg/signinum 0.4.2); see oracle_internal.h.  Only the tests, the smoke
check and the benchmark's CPU-baseline leg load it; the product package never
does.  build() compiles it with oracle/Makefile into oracle/_build/.
"""
import ctypes
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"

FMT_BPP = {0: 1, 1: 3, 2: 4, 3: 2, 4: 6, 5: 8}


class OracleInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in
                ("width", "height", "components", "bit_depth", "levels", "tiles", "ht", "reversible", "mct")]


class OracleError(Exception):
    def __init__(self, status, message):
        super().__init__(f"[{status}] {message}")
        self.status = status


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = ctypes.CDLL(str(LIB))
        L.oracle_last_error.restype = ctypes.c_char_p
        L.oracle_inspect.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(OracleInfo)]
        L.oracle_decode.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_int, ctypes.c_uint32,
                                    ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                    ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint32),
                                    ctypes.POINTER(ctypes.c_uint32)]
        L.oracle_ht_block_decode.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t,
                                             ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                             ctypes.c_int, ctypes.c_void_p]
        L.oracle_subband_coefficients.restype = ctypes.c_long
        L.oracle_subband_coefficients.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32,
                                                  ctypes.c_void_p, ctypes.c_size_t]
        L.oracle_tables.argtypes = [ctypes.c_void_p] * 4
        L.oracle_ebcot_tables.argtypes = [ctypes.c_void_p] * 6
        L.oracle_decode_batch.restype = ctypes.c_long
        L.oracle_decode_batch.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t),
                                          ctypes.c_size_t, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                          ctypes.POINTER(ctypes.c_size_t), ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_int)]
        _lib = L
    return _lib


def _buf(data):
    return np.frombuffer(bytes(data), dtype=np.uint8) if not isinstance(data, np.ndarray) else data


def inspect(data):
    a = _buf(data)
    i = OracleInfo()
    st = lib().oracle_inspect(a.ctypes.data, a.nbytes, ctypes.byref(i))
    if st:
        raise OracleError(st, lib().oracle_last_error().decode())
    return i


def decode(data, fmt, kind=0, roi=(0, 0, 0, 0), denom=1):
    """Decoded pixels (tight bytes), width and height; raises OracleError."""
    a = _buf(data)
    info = inspect(a)
    cap = max(1, info.width * info.height * FMT_BPP.get(fmt, 8))
    out = np.zeros(cap, dtype=np.uint8)
    w, h = ctypes.c_uint32(), ctypes.c_uint32()
    st = lib().oracle_decode(a.ctypes.data, a.nbytes, fmt, kind, roi[0], roi[1], roi[2], roi[3], denom,
                             out.ctypes.data, cap, ctypes.byref(w), ctypes.byref(h))
    if st:
        raise OracleError(st, lib().oracle_last_error().decode())
    return out[: w.value * h.value * FMT_BPP[fmt]].tobytes(), w.value, h.value


def tables():
    v0 = np.zeros(1024, np.uint16)
    v1 = np.zeros(1024, np.uint16)
    u0 = np.zeros(320, np.uint16)
    u1 = np.zeros(256, np.uint16)
    lib().oracle_tables(v0.ctypes.data, v1.ctypes.data, u0.ctypes.data, u1.ctypes.data)
    return v0, v1, u0, u1


def ebcot_tables():
    """Classic Tier-1 tables: zero-coding (LL/LH, HL, HH), sign label, sign
    xor (256 u8 each) and the MQ probability records (235 bytes)."""
    bufs = [np.zeros(256, np.uint8) for _ in range(5)] + [np.zeros(235, np.uint8)]
    lib().oracle_ebcot_tables(*[b.ctypes.data for b in bufs])
    return bufs


def decode_batch(datas, fmt, workers=0):
    """CPU tile batch (decode_tiles_into restated); returns (outputs, lowest failing index or -1)."""
    n = len(datas)
    arrs = [_buf(d) for d in datas]
    outs = []
    for a in arrs:
        i = inspect(a)
        outs.append(np.zeros(max(1, i.width * i.height * FMT_BPP[fmt]), np.uint8))
    ptrs = (ctypes.c_void_p * n)(*[a.ctypes.data for a in arrs])
    lens = (ctypes.c_size_t * n)(*[a.nbytes for a in arrs])
    optr = (ctypes.c_void_p * n)(*[o.ctypes.data for o in outs])
    caps = (ctypes.c_size_t * n)(*[o.nbytes for o in outs])
    per = (ctypes.c_int * n)()
    first = lib().oracle_decode_batch(ptrs, lens, n, fmt, optr, caps, workers, per)
    return outs, first
