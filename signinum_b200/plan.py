"""Device-resident batch plans (sgn_plan_* in include/signinum_j2k_cuda.h).

A plan parses a batch once, keeps its codestreams and descriptor tables in
device memory and owns its output surfaces; execute() replays the decode.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np

from . import _native
from ._native import SgnRequest, SgnSurface
from .j2k_cuda import Error, _check, _Context, _as_u8


class Plan:
    def __init__(self, inputs: Sequence, fmt: int, requests: Optional[Sequence[SgnRequest]] = None,
                 ctx: Optional[_Context] = None, contiguous: Optional[np.ndarray] = None,
                 offsets: Optional[Sequence[int]] = None):
        """inputs: codestreams; or pass `contiguous` (one buffer, e.g. pinned)
        with per-tile `offsets` into it and `inputs` as the lengths."""
        self.ctx = ctx or _Context.default()
        lib = _native.cuda_lib()
        if contiguous is not None:
            base = contiguous.ctypes.data
            n = len(offsets)
            ptrs = (ctypes.c_void_p * n)(*[base + o for o in offsets])
            lens = (ctypes.c_size_t * n)(*list(inputs))
            self._keep = contiguous
        else:
            arrs = [_as_u8(d) for d in inputs]
            n = len(arrs)
            ptrs = (ctypes.c_void_p * n)(*[a.ctypes.data for a in arrs])
            lens = (ctypes.c_size_t * n)(*[a.nbytes for a in arrs])
            self._keep = arrs
        self.n = n
        reqs = (SgnRequest * n)(*requests) if requests is not None else None
        per = (ctypes.c_int32 * n)()
        h = ctypes.c_void_p()
        _check(lib.sgn_plan_create(self.ctx.handle, ptrs, lens, n, int(fmt), reqs, ctypes.byref(h), per))
        self.handle = h
        self.parse_status = list(per)
        self.launches = lib.sgn_plan_kernel_launches(h)

    def execute_async(self):
        _check(_native.cuda_lib().sgn_plan_execute_async(self.ctx.handle, self.handle))

    def wait(self):
        per = (ctypes.c_int32 * self.n)()
        first = ctypes.c_size_t()
        st = _native.cuda_lib().sgn_plan_wait(self.ctx.handle, self.handle, per, ctypes.byref(first))
        return st, list(per)

    def autotune(self, reps: int = 5) -> dict:
        """Times candidate launch shapes on this plan's data and keeps the fastest
        (sgn_plan_autotune); returns the chosen shape and stage times."""
        from ._native import SgnTuneReport

        r = SgnTuneReport()
        _check(_native.cuda_lib().sgn_plan_autotune(self.ctx.handle, self.handle, reps, ctypes.byref(r)))
        return {n: getattr(r, n) for n, _ in SgnTuneReport._fields_}

    def set_launch_shape(self, vlc_threads=128, ms_warps=8, ms_blocks_per_grab=0, dwt_queue=0):
        _check(_native.cuda_lib().sgn_plan_set_launch_shape(self.ctx.handle, self.handle, vlc_threads, ms_warps,
                                                            ms_blocks_per_grab, dwt_queue))

    def set_tile_shape(self, idwt_seg_shift=0, pack_seg_shift=0):
        """Rows per IDWT / pack work unit: the base rule scaled by 2^shift."""
        _check(_native.cuda_lib().sgn_plan_set_tile_shape(self.ctx.handle, self.handle, idwt_seg_shift,
                                                          pack_seg_shift))

    def set_cleanup_form(self, fused=2):
        """HT cleanup passes: 0 the VLC then the MagSgn kernel, 1 both in one
        kernel (a CTA per code block), 2 chosen by block count."""
        _check(_native.cuda_lib().sgn_plan_set_cleanup_form(self.ctx.handle, self.handle, fused))

    def execute_timed(self):
        """Per-stage milliseconds: HT VLC pass, HT MagSgn pass, HT refinement, IDWT levels,
        last level + pack, total."""
        ms = (ctypes.c_float * 6)()
        _check(_native.cuda_lib().sgn_plan_execute_timed(self.ctx.handle, self.handle, ms))
        return list(ms)

    def surfaces(self):
        outs = (SgnSurface * self.n)()
        _check(_native.cuda_lib().sgn_plan_surfaces(self.handle, outs, self.n))
        return list(outs)

    def download(self, i: int) -> bytes:
        s = self.surfaces()[i]
        out = np.zeros(max(1, s.pitch_bytes * s.height), np.uint8)
        _check(_native.cuda_lib().sgn_surface_download(self.ctx.handle, ctypes.byref(s), out.ctypes.data, out.nbytes,
                                                        s.pitch_bytes))
        return out[: s.pitch_bytes * s.height].tobytes()

    def destroy(self):
        if self.handle:
            _native.cuda_lib().sgn_plan_destroy(self.ctx.handle, self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


__all__ = ["Plan", "Error"]
