"""Python face of the CUDA decode path, mirroring the reference's
signinum-j2k-cuda adapter (crates/signinum-j2k-cuda/src/lib.rs:21-27).

    J2kDecoder(bytes).decode_to_device(PixelFormat.Rgb8, BackendRequest.Cuda)
    Codec.decode_tiles_to_device([tile0, tile1, ...], PixelFormat.Rgb8, BackendRequest.Cuda)

Names, argument meaning and error predicates follow the reference:
J2kDecoder (decoder.rs:17-280), Codec (codec.rs:18-210), CudaSession
(session.rs:11-39), Surface / CudaSurface (surface.rs:19-127), Error
(error.rs:7-41).  BackendRequest.Cuda decodes on the GPU through the C ABI
of libsigninum_j2k_cuda.so.  Cpu and Auto keep the reference adapter's
host-surface branch (wrap_surface, crates/signinum-j2k-cuda/src/runtime.rs:19-48):
the caller's host decoder (the reference's own CPU J2kDecoder, registered
with set_host_decoder) produces the bytes and the surface is a host one;
no CUDA context is created for them.  This package carries no host decoder
of its own, so without a registered one Cpu and Auto raise an Error whose
is_host_backend() is true.  Metal is an unsupported backend.
"""
from __future__ import annotations

import ctypes
import enum
from dataclasses import dataclass
from typing import Callable, Optional, Sequence

import numpy as np

from . import _native
from ._native import SgnInfo, SgnRequest, SgnSurface

OK = 0
ERR_UNSUPPORTED = 1
ERR_BUFFER = 2
ERR_TRUNCATED = 3
ERR_DECODE = 4
ERR_REGION = 5
ERR_CUDA_UNAVAILABLE = 6
ERR_CUDA_RUNTIME = 7
ERR_UNSUPPORTED_BACKEND = 8
ERR_INVALID_ARGUMENT = 9
ERR_OUT_OF_MEMORY = 10
ERR_HOST_BACKEND = 11


class BackendRequest(enum.IntEnum):
    """signinum_core::BackendRequest (crates/signinum-core/src/backend.rs:15-22)."""
    Auto = 0
    Cpu = 1
    Metal = 2
    Cuda = 3


class BackendKind(enum.IntEnum):
    Cpu = 0
    Cuda = 3


class PixelFormat(enum.IntEnum):
    """signinum_core::PixelFormat values used on this path."""
    Gray8 = 0
    Rgb8 = 1
    Rgba8 = 2
    Gray16 = 3
    Rgb16 = 4
    Rgba16 = 5

    def bytes_per_pixel(self) -> int:
        return (1, 3, 4, 2, 6, 8)[self]


class Downscale(enum.Enum):
    """signinum_core::Downscale (crates/signinum-core/src/scale.rs:5-20)."""
    None_ = 1
    Half = 2
    Quarter = 4
    Eighth = 8

    def denominator(self) -> int:
        return self.value


@dataclass(frozen=True)
class Rect:
    """signinum_core::Rect (crates/signinum-core/src/types.rs:46-84)."""
    x: int
    y: int
    w: int
    h: int

    @staticmethod
    def full(dims) -> "Rect":
        return Rect(0, 0, dims[0], dims[1])

    def is_within(self, dims) -> bool:
        return self.x + self.w <= dims[0] and self.y + self.h <= dims[1]

    def scaled_covering(self, scale: Downscale) -> "Rect":
        d = scale.denominator()
        x0, y0 = self.x // d, self.y // d
        x1, y1 = -(-(self.x + self.w) // d), -(-(self.y + self.h) // d)
        return Rect(x0, y0, max(0, x1 - x0), max(0, y1 - y0))


class Error(Exception):
    """crates/signinum-j2k-cuda/src/error.rs:7-41, carrying the C status code."""

    def __init__(self, status: int, message: str = ""):
        super().__init__(f"[{status}] {message}")
        self.status = status
        self.message = message

    def is_unsupported(self) -> bool:
        return self.status in (ERR_UNSUPPORTED, ERR_UNSUPPORTED_BACKEND, ERR_CUDA_UNAVAILABLE)

    def is_not_implemented(self) -> bool:
        return self.status == ERR_UNSUPPORTED

    def is_truncated(self) -> bool:
        return self.status == ERR_TRUNCATED

    def is_buffer_error(self) -> bool:
        return self.status == ERR_BUFFER

    def is_invalid_region(self) -> bool:
        return self.status == ERR_REGION

    def is_host_backend(self) -> bool:
        """Cpu / Auto request with no host decoder registered: the adapter's
        host branch, which this package does not implement."""
        return self.status == ERR_HOST_BACKEND


def _check(status: int):
    if status != OK:
        raise Error(status, _native.last_error())


def _as_u8(data) -> np.ndarray:
    if isinstance(data, np.ndarray):
        return np.ascontiguousarray(data).view(np.uint8).reshape(-1)
    return np.frombuffer(bytes(data) if not isinstance(data, (bytes, bytearray, memoryview)) else data,
                         dtype=np.uint8)


class CudaSession:
    """Lazily owns a CUDA context on one device (session.rs:11-39)."""

    def __init__(self, device: int = 0):
        self._device = device
        self._ctx = None
        self._submissions = 0

    def submissions(self) -> int:
        return self._submissions

    def is_runtime_initialized(self) -> bool:
        return self._ctx is not None

    def record_submit(self):
        self._submissions += 1

    def cuda_context(self):
        if self._ctx is None:
            self._ctx = _Context.open(self._device)
        return self._ctx


class _Context:
    """Owner of one sgn_ctx; shared by the surfaces it produced."""

    _default = {}

    def __init__(self, handle, device):
        self.handle = handle
        self.device = device

    @classmethod
    def open(cls, device: int) -> "_Context":
        lib = _native.cuda_lib()
        h = ctypes.c_void_p()
        _check(lib.sgn_ctx_create(device, ctypes.byref(h)))
        return cls(h, device)

    @classmethod
    def default(cls, device: int = 0) -> "_Context":
        if device not in cls._default:
            cls._default[device] = cls.open(device)
        return cls._default[device]

    def stream(self) -> int:
        return _native.cuda_lib().sgn_ctx_stream(self.handle) or 0

    def __del__(self):
        try:
            if self.handle:
                _native.cuda_lib().sgn_ctx_destroy(self.handle)
        except Exception:
            pass


@dataclass
class CudaSurfaceStats:
    kernel_dispatches_: int

    def kernel_dispatches(self) -> int:
        return self.kernel_dispatches_


class CudaSurface:
    def __init__(self, surface: "Surface"):
        self._s = surface

    def device_ptr(self) -> int:
        return self._s._raw.device_ptr

    def stats(self) -> CudaSurfaceStats:
        return CudaSurfaceStats(self._s._raw.kernel_dispatches)


class Surface:
    """A decoded tile (surface.rs:55-127); tight rows.  Device storage for
    BackendRequest.Cuda, host storage for the Cpu / Auto branch."""

    def __init__(self, raw: SgnSurface, ctx: Optional[_Context], host: Optional[bytes] = None):
        self._raw = raw
        self._ctx = ctx
        self._host = host

    @classmethod
    def from_host(cls, data: bytes, dims, fmt: PixelFormat) -> "Surface":
        raw = SgnSurface()
        raw.width, raw.height = dims
        raw.format = int(fmt)
        raw.backend = int(BackendKind.Cpu)
        raw.pitch_bytes = dims[0] * PixelFormat(fmt).bytes_per_pixel()
        return cls(raw, None, bytes(data))

    def backend_kind(self) -> BackendKind:
        return BackendKind.Cpu if self._host is not None else BackendKind.Cuda

    def dimensions(self):
        return (self._raw.width, self._raw.height)

    def pixel_format(self) -> PixelFormat:
        return PixelFormat(self._raw.format)

    def pitch_bytes(self) -> int:
        return self._raw.pitch_bytes

    def byte_len(self) -> int:
        return self._raw.pitch_bytes * self._raw.height

    def as_host_bytes(self):
        return self._host

    def cuda_surface(self) -> Optional[CudaSurface]:
        return CudaSurface(self) if self._host is None else None

    def download_into(self, out, stride: int):
        buf = out if isinstance(out, np.ndarray) else np.frombuffer(out, dtype=np.uint8)
        if self._host is not None:
            # Surface::download_into for host storage (surface.rs:78-92).
            row, h = self.pitch_bytes(), self._raw.height
            if h and (stride < row or buf.nbytes < stride * (h - 1) + row):
                raise Error(ERR_BUFFER, "output buffer too small for the surface")
            src = np.frombuffer(self._host, np.uint8)
            for y in range(h):
                buf[y * stride:y * stride + row] = src[y * row:(y + 1) * row]
            return
        _check(_native.cuda_lib().sgn_surface_download(self._ctx.handle, ctypes.byref(self._raw),
                                                        buf.ctypes.data, buf.nbytes, stride))

    def to_bytes(self) -> bytes:
        if self._host is not None:
            return self._host
        out = np.zeros(self.byte_len(), dtype=np.uint8)
        self.download_into(out, self.pitch_bytes())
        return out.tobytes()

    def free(self):
        if self._host is None and self._raw.device_ptr:
            _native.cuda_lib().sgn_surface_free(self._ctx.handle, ctypes.byref(self._raw))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# The host decoder of the Cpu / Auto branch: a callable
# (codestream bytes, PixelFormat, SgnRequest) -> (pixels bytes, (width, height)).
HostDecoder = Callable[[bytes, PixelFormat, SgnRequest], tuple]
_host_decoder: Optional[HostDecoder] = None


def set_host_decoder(fn: Optional[HostDecoder]) -> Optional[HostDecoder]:
    """Registers the decoder that serves BackendRequest.Cpu and .Auto (the
    reference's CPU J2kDecoder in a signinum process); returns the previous
    one.  None removes it."""
    global _host_decoder
    prev, _host_decoder = _host_decoder, fn
    return prev


def _host_branch(data, fmt: PixelFormat, req: SgnRequest, backend: BackendRequest) -> Surface:
    """wrap_surface's Cpu | Auto arm (runtime.rs:19-48): host bytes in a host
    surface; CUDA is not touched."""
    if PixelFormat(fmt) == PixelFormat.Rgba16:
        raise Error(ERR_UNSUPPORTED, "Rgba16 output is not supported")
    if _host_decoder is None:
        raise Error(ERR_HOST_BACKEND, f"backend request {backend.name} takes the host-surface branch and no host "
                                      "decoder is registered (set_host_decoder); this package decodes on CUDA only")
    pixels, dims = _host_decoder(bytes(_as_u8(data)), PixelFormat(fmt), req)
    return Surface.from_host(pixels, dims, PixelFormat(fmt))


def _request(kind=0, roi: Optional[Rect] = None, scale: Optional[Downscale] = None) -> SgnRequest:
    r = SgnRequest()
    r.kind = kind
    if roi is not None:
        r.x, r.y, r.w, r.h = roi.x, roi.y, roi.w, roi.h
    r.downscale = scale.denominator() if scale is not None else 1
    return r


def _decode_one(ctx: _Context, data, fmt: PixelFormat, req: SgnRequest, backend: BackendRequest) -> Surface:
    arr = _as_u8(data)
    out = SgnSurface()
    _check(_native.cuda_lib().sgn_j2k_decode_to_device(ctx.handle, arr.ctypes.data, arr.nbytes, int(fmt),
                                                         ctypes.byref(req), int(backend), ctypes.byref(out)))
    return Surface(out, ctx)


def _validate_backend(backend: BackendRequest):
    """validate_surface_request (runtime.rs:52-57)."""
    if BackendRequest(backend) == BackendRequest.Metal:
        raise Error(ERR_UNSUPPORTED_BACKEND, "backend request Metal is not supported by signinum-j2k-cuda")


def _is_host(backend: BackendRequest) -> bool:
    return BackendRequest(backend) in (BackendRequest.Cpu, BackendRequest.Auto)


@dataclass
class Info:
    dimensions: tuple
    components: int
    bit_depth: int
    resolution_levels: int
    tiles: int
    ht: bool
    reversible: bool
    mct: bool


def inspect(data) -> Info:
    arr = _as_u8(data)
    i = SgnInfo()
    _check(_native.cuda_lib().sgn_j2k_inspect(arr.ctypes.data, arr.nbytes, ctypes.byref(i)))
    return Info((i.width, i.height), i.components, i.bit_depth, i.levels + 1, i.tiles, bool(i.ht),
                bool(i.reversible), bool(i.mct))


class J2kDecoder:
    """crates/signinum-j2k-cuda/src/decoder.rs:17-280."""

    def __init__(self, data):
        self._data = _as_u8(data)
        self._info = inspect(self._data)

    def info(self) -> Info:
        return self._info

    def _decode(self, fmt, req: SgnRequest, backend, session: Optional[CudaSession]) -> Surface:
        _validate_backend(backend)
        if session is not None:
            session.record_submit()
        if _is_host(backend):
            return _host_branch(self._data, fmt, req, backend)
        ctx = session.cuda_context() if session is not None else _Context.default()
        return _decode_one(ctx, self._data, fmt, req, backend)

    def decode_to_device(self, fmt: PixelFormat, backend: BackendRequest, session: Optional[CudaSession] = None):
        return self._decode(fmt, _request(0), backend, session)

    def decode_region_to_device(self, fmt, roi: Rect, backend, session=None):
        return self._decode(fmt, _request(1, roi), backend, session)

    def decode_scaled_to_device(self, fmt, scale: Downscale, backend, session=None):
        return self._decode(fmt, _request(2, None, scale), backend, session)

    def decode_region_scaled_to_device(self, fmt, roi: Rect, scale: Downscale, backend, session=None):
        return self._decode(fmt, _request(3, roi, scale), backend, session)

    # ImageDecodeSubmit: the submission is ready when the call returns.
    def submit_to_device(self, session: CudaSession, fmt, backend):
        return self.decode_to_device(fmt, backend, session)


class TileBatchError(Error):
    """crates/signinum-core/src/batch.rs:49-67: the lowest failing index."""

    def __init__(self, index: int, status: int, message: str):
        super().__init__(status, message)
        self.index = index


class Codec:
    """crates/signinum-j2k-cuda/src/codec.rs:18-210."""

    @staticmethod
    def decode_tile_to_device(data, fmt, backend, session: Optional[CudaSession] = None):
        return J2kDecoder(data).decode_to_device(fmt, backend, session)

    @staticmethod
    def decode_tile_region_to_device(data, fmt, roi, backend, session=None):
        return J2kDecoder(data).decode_region_to_device(fmt, roi, backend, session)

    @staticmethod
    def decode_tile_scaled_to_device(data, fmt, scale, backend, session=None):
        return J2kDecoder(data).decode_scaled_to_device(fmt, scale, backend, session)

    @staticmethod
    def decode_tile_region_scaled_to_device(data, fmt, roi, scale, backend, session=None):
        return J2kDecoder(data).decode_region_scaled_to_device(fmt, roi, scale, backend, session)

    @staticmethod
    def decode_tiles_to_device(inputs: Sequence, fmt: PixelFormat, backend: BackendRequest,
                               requests: Optional[Sequence[SgnRequest]] = None,
                               session: Optional[CudaSession] = None):
        """TileBatchDecodeManyDevice::decode_tiles_to_device: one surface per
        input, order preserved; raises TileBatchError for the lowest failing
        index."""
        _validate_backend(backend)
        if _is_host(backend):
            surfaces = []
            for i, d in enumerate(inputs):
                try:
                    surfaces.append(_host_branch(d, fmt, requests[i] if requests is not None else _request(0),
                                                 backend))
                except Error as e:
                    raise TileBatchError(i, e.status, e.message) from e
            return surfaces
        ctx = session.cuda_context() if session is not None else _Context.default()
        arrs = [_as_u8(d) for d in inputs]
        n = len(arrs)
        ptrs = (ctypes.c_void_p * n)(*[a.ctypes.data for a in arrs])
        lens = (ctypes.c_size_t * n)(*[a.nbytes for a in arrs])
        outs = (SgnSurface * n)()
        per = (ctypes.c_int32 * n)()
        first = ctypes.c_size_t()
        reqs = None
        if requests is not None:
            reqs = (SgnRequest * n)(*requests)
        st = _native.cuda_lib().sgn_j2k_decode_tiles_to_device(ctx.handle, ptrs, lens, n, int(fmt), reqs,
                                                                int(backend), outs, per, ctypes.byref(first))
        surfaces = [Surface(outs[i], ctx) for i in range(n)]
        if st != OK:
            idx = first.value if first.value < n else 0
            raise TileBatchError(idx, per[idx] if n else st, _native.last_error())
        return surfaces


def dicom_frames(data, limit: Optional[int] = None):
    """JPEG 2000 frames of a DICOM file's encapsulated Pixel Data
    (extract_dicom_encapsulated_frames, crates/signinum-j2k-metal/src/dicom.rs:22-95),
    as a list of bytes."""
    arr = _as_u8(data)
    lim = ctypes.c_size_t(-1).value if limit is None else limit
    n, total = ctypes.c_size_t(), ctypes.c_size_t()
    lib = _native.cuda_lib()
    _check(lib.sgn_dicom_frames(arr.ctypes.data, arr.nbytes, lim, None, 0, None, None, 0, ctypes.byref(n),
                                ctypes.byref(total)))
    out = np.zeros(max(1, total.value), np.uint8)
    offs = (ctypes.c_uint64 * max(1, n.value))()
    lens = (ctypes.c_uint64 * max(1, n.value))()
    _check(lib.sgn_dicom_frames(arr.ctypes.data, arr.nbytes, lim, out.ctypes.data, out.nbytes, offs, lens, n.value,
                                ctypes.byref(n), ctypes.byref(total)))
    return [out[offs[i]:offs[i] + lens[i]].tobytes() for i in range(n.value)]
