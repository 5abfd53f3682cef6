"""Backend routing at the boundary, mirroring the reference adapter's tests
(crates/signinum-j2k-cuda/tests/host_surface.rs) on a host with no GPU.

wrap_surface (crates/signinum-j2k-cuda/src/runtime.rs:19-48) serves
BackendRequest::Cpu and ::Auto with a host surface of the CPU decoder's
bytes and never initialises CUDA (session.rs:32-38); ::Cuda goes to the
device; ::Metal is an unsupported backend.  Here the C ABI answers Cpu and
Auto with SGN_ERR_HOST_BACKEND before any CUDA call, and the Python mirror
keeps the adapter's host branch, with the caller's host decoder producing
the bytes (the tests register the oracle, the restated reference CPU
decoder, in that role).
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle
from signinum_b200 import (BackendKind, BackendRequest, Codec, CudaSession, Error, J2kDecoder, PixelFormat, _native,
                           encode, set_host_decoder)
from signinum_b200._native import SgnRequest, SgnSurface


def _oracle_host_decoder(data, fmt, req):
    got, w, h = oracle.decode(data, int(fmt), req.kind, (req.x, req.y, req.w, req.h), req.downscale or 1)
    return got, (w, h)


@pytest.fixture
def host_decoder():
    prev = set_host_decoder(_oracle_host_decoder)
    yield
    set_host_decoder(prev)


def _fixture():
    # host_surface.rs:19-27: a 4x4 HT gray tile, pixels 0..15, one level.
    px = np.arange(16, dtype=np.uint8)
    return encode.encode_lossless(px, 4, 4, 1, 8, levels=1, cb_exp=2, use_mct=False), px


def test_submit_to_device_auto_does_not_initialize_cuda_runtime(host_decoder):
    # host_surface.rs:203-221
    cs, px = _fixture()
    session = CudaSession()
    surface = J2kDecoder(cs).submit_to_device(session, PixelFormat.Gray8, BackendRequest.Auto)
    assert surface.backend_kind() == BackendKind.Cpu
    assert surface.as_host_bytes() == px.tobytes()
    assert surface.cuda_surface() is None
    assert session.submissions() == 1
    assert not session.is_runtime_initialized()


def test_cpu_request_returns_host_surface(host_decoder):
    # host_surface.rs:29-57: Cpu gives a host surface with tight rows.
    t = encode.config0(keep_pixels=True).tiles[0]
    session = CudaSession()
    s = J2kDecoder(t.codestream).decode_to_device(PixelFormat.Rgb8, BackendRequest.Cpu, session)
    assert s.backend_kind() == BackendKind.Cpu
    assert s.pitch_bytes() == 256 * 3 and s.byte_len() == 256 * 256 * 3
    stride = 256 * 3 + 5
    out = np.zeros(stride * 256, np.uint8)
    s.download_into(out, stride)
    assert out.reshape(256, stride)[:, :256 * 3].tobytes() == t.pixels.tobytes()
    with pytest.raises(Error) as e:
        s.download_into(np.zeros(10, np.uint8), stride)
    assert e.value.is_buffer_error()
    assert not session.is_runtime_initialized()


def test_auto_tile_batch_takes_the_host_branch_in_order(host_decoder):
    w = encode.config2(n=5)
    surfaces = Codec.decode_tiles_to_device([t.codestream for t in w.tiles], PixelFormat.Rgb8, BackendRequest.Auto)
    assert [s.backend_kind() for s in surfaces] == [BackendKind.Cpu] * 5
    for t, s in zip(w.tiles, surfaces):
        assert s.dimensions() == (t.width, t.height)


def test_host_branch_without_a_host_decoder_is_reported_not_decoded():
    prev = set_host_decoder(None)
    try:
        cs, _ = _fixture()
        session = CudaSession()
        for b in (BackendRequest.Cpu, BackendRequest.Auto):
            with pytest.raises(Error) as e:
                J2kDecoder(cs).decode_to_device(PixelFormat.Gray8, b, session)
            assert e.value.is_host_backend() and not e.value.is_unsupported()
        assert not session.is_runtime_initialized()
    finally:
        set_host_decoder(prev)


def test_metal_is_an_unsupported_backend():
    cs, _ = _fixture()
    session = CudaSession()
    with pytest.raises(Error) as e:
        J2kDecoder(cs).decode_to_device(PixelFormat.Gray8, BackendRequest.Metal, session)
    assert e.value.is_unsupported()
    assert not session.is_runtime_initialized()


def test_c_abi_answers_host_backends_before_any_cuda_call():
    """No context (NULL) and no GPU needed: Cpu / Auto return
    SGN_ERR_HOST_BACKEND, Metal SGN_ERR_UNSUPPORTED_BACKEND, before the
    context is even looked at."""
    lib = _native.cuda_lib()
    cs, _ = _fixture()
    arr = np.frombuffer(cs, np.uint8)
    req = SgnRequest(0, 0, 0, 0, 0, 1)
    out = SgnSurface()
    for backend, want in ((0, 11), (1, 11), (2, 8)):
        st = lib.sgn_j2k_decode_to_device(None, arr.ctypes.data, arr.nbytes, 0, ctypes.byref(req), backend,
                                          ctypes.byref(out))
        assert st == want, (backend, st)
        n = 1
        ptrs = (ctypes.c_void_p * n)(arr.ctypes.data)
        lens = (ctypes.c_size_t * n)(arr.nbytes)
        outs = (SgnSurface * n)()
        per = (ctypes.c_int32 * n)()
        first = ctypes.c_size_t()
        st = lib.sgn_j2k_decode_tiles_to_device(None, ptrs, lens, n, 0, None, backend, outs, per, ctypes.byref(first))
        assert st == want, (backend, st)
