"""The C-ABI libraries load and export every declared entry point (CPU)."""
import ctypes
import pathlib
import re

import numpy as np

from signinum_b200 import _native, encode, inspect

INCLUDE = pathlib.Path(__file__).resolve().parent.parent / "include"


def _declared(header):
    text = re.sub(r"/\*.*?\*/", "", (INCLUDE / header).read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(sgn_[a-z0-9_]+)\s*\(", text)))


def test_cuda_library_exports_header_symbols():
    lib = ctypes.CDLL(str(_native.CUDA_LIB))
    names = _declared("signinum_j2k_cuda.h")
    assert "sgn_j2k_decode_to_device" in names and "sgn_j2k_decode_tiles_to_device" in names
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) <= set(_native.CUDA_SIGNATURES), set(names) - set(_native.CUDA_SIGNATURES)


def test_encode_library_exports_header_symbols():
    lib = ctypes.CDLL(str(_native.ENCODE_LIB))
    for n in _declared("signinum_j2k_encode.h"):
        assert hasattr(lib, n), n


def test_inspect_runs_on_host():
    t = encode.config0().tiles[0]
    info = inspect(t.codestream)
    assert info.dimensions == (256, 256)
    assert info.components == 3 and info.bit_depth == 8 and info.ht and info.reversible and info.mct
    assert info.resolution_levels == 6


def test_inspect_rejects_garbage():
    from signinum_b200 import Error

    try:
        inspect(b"\x00\x01\x02\x03")
    except Error as e:
        assert e.status == 1 and e.is_unsupported()  # not a JP2 container or raw codestream
    else:
        raise AssertionError("garbage accepted")


def test_context_creation_reports_unavailable_without_gpu():
    import torch

    if torch.cuda.is_available():
        return
    h = ctypes.c_void_p()
    st = _native.cuda_lib().sgn_ctx_create(0, ctypes.byref(h))
    assert st == 6  # SGN_ERR_CUDA_UNAVAILABLE -> Error::is_unsupported()
