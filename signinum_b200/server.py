"""Serving loop over the CUDA decode path: continuous batching of tile requests.

Wraps sgn_server_* (include/signinum_j2k_cuda.h).  Codestreams are
registered once and stay resident on the device; requests (full, region,
reduced resolution, region at reduced resolution) are queued by `submit`,
batched by the native dispatcher as CUDA streams and device memory free up,
and come back from `poll` with their surface, status and latency.  The
reference has no serving loop; its adapter decodes one call at a time
(crates/signinum-j2k-cuda/src/codec.rs:18-210), and every request here
decodes exactly as that call would.
"""
import ctypes
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from . import _native
from ._native import SgnServerConfig, SgnServerResult, SgnServerStats, SgnSurface
from .j2k_cuda import Downscale, PixelFormat, Rect, Surface, _as_u8, _check, _Context, _request

REQ_FULL, REQ_REGION, REQ_SCALED, REQ_REGION_SCALED = 0, 1, 2, 3


class ServerSurface(Surface):
    """A result surface; freed through the server without a device sync."""

    def __init__(self, raw: SgnSurface, ctx: _Context, server: "Server"):
        super().__init__(raw, ctx)
        self._server = server

    def free(self):
        if self._raw.device_ptr and self._server._h:
            _native.cuda_lib().sgn_server_surface_free(self._server._h, ctypes.byref(self._raw))


@dataclass
class Result:
    ticket: int
    status: int
    batch_tiles: int
    latency_ms: float
    queue_ms: float
    surface: Optional[ServerSurface]


class Server:
    def __init__(self, ctx: Optional[_Context] = None, device_budget_bytes: int = 16 << 30,
                 resident_capacity_bytes: int = 1 << 30, max_batch_tiles: int = 512, slots: int = 3,
                 max_batch_samples: int = 0):
        self.ctx = ctx or _Context.default(0)
        cfg = SgnServerConfig(device_budget_bytes, resident_capacity_bytes, max_batch_tiles, slots, 0,
                              max_batch_samples)
        h = ctypes.c_void_p()
        _check(_native.cuda_lib().sgn_server_create(self.ctx.handle, ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h

    def register(self, data) -> int:
        arr = _as_u8(data)
        tid = ctypes.c_uint32()
        _check(_native.cuda_lib().sgn_server_register(self._h, arr.ctypes.data, arr.nbytes, ctypes.byref(tid)))
        return tid.value

    def submit(self, tile_id: int, fmt: PixelFormat = PixelFormat.Rgb8, roi: Optional[Rect] = None,
               scale: Optional[Downscale] = None) -> int:
        kind = REQ_FULL
        if roi is not None and scale is not None and scale != Downscale.None_:
            kind = REQ_REGION_SCALED
        elif roi is not None:
            kind = REQ_REGION
        elif scale is not None and scale != Downscale.None_:
            kind = REQ_SCALED
        req = _request(kind, roi, scale)
        t = ctypes.c_uint64()
        _check(_native.cuda_lib().sgn_server_submit(self._h, tile_id, int(fmt), ctypes.byref(req), ctypes.byref(t)))
        return t.value

    def poll(self, max_results: int = 1024, timeout_ms: int = 0) -> List[Result]:
        buf = (SgnServerResult * max_results)()
        n = ctypes.c_size_t()
        _check(_native.cuda_lib().sgn_server_poll(self._h, buf, max_results, ctypes.byref(n), timeout_ms))
        out = []
        for r in buf[: n.value]:
            raw = SgnSurface()
            ctypes.pointer(raw)[0] = r.surface
            surf = ServerSurface(raw, self.ctx, self) if r.surface.device_ptr else None
            out.append(Result(r.ticket, r.status, r.batch_tiles, r.latency_ms, r.queue_ms, surf))
        return out

    def stats(self) -> dict:
        s = SgnServerStats()
        _check(_native.cuda_lib().sgn_server_stats_get(self._h, ctypes.byref(s)))
        return {n: getattr(s, n) for n, _ in SgnServerStats._fields_}

    def close(self):
        if self._h:
            _native.cuda_lib().sgn_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def collect(server: Server, tickets, timeout_s: float = 30.0) -> dict:
    """Polls until every ticket has a result; returns {ticket: Result}."""
    import time

    want = set(tickets)
    got = {}
    end = time.perf_counter() + timeout_s
    while want - got.keys():
        if time.perf_counter() > end:
            raise TimeoutError(f"{len(want - got.keys())} requests without a result")
        for r in server.poll(1024, 50):
            got[r.ticket] = r
    return got


__all__ = ["Server", "Result", "ServerSurface", "collect", "np"]
