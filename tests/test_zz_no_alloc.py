"""The HT decode entry point that allocates nothing, checked against the
existing decode path.

Some callers of this library cannot call cudaMalloc: a host framework whose
caching allocator owns all of the GPU's memory, a decoder plugin that is
handed its input and output buffers and may create none of its own, and
real-time loops that must not allocate once they run.
sgn_ht_decode_blocks_noalloc serves them: inputs and outputs are the
caller's device memory and its scratch is a fixed static device array.  Its
coefficients must equal, bit for bit (the reversible path is integer
arithmetic, so the tolerance is zero), the HT stage output of the regular
plan path for the same codestream, on two calls in a row that share that
static scratch.

This file is named to be collected last, so a failing run that stops at the
first failure has already run every other test.
"""
import ctypes
import json
import pathlib

import numpy as np
import pytest

from signinum_b200 import PixelFormat, _native, encode
from signinum_b200._native import SgnHtBlock
from signinum_b200.plan import Plan

pytestmark = pytest.mark.gpu

GOLDEN = pathlib.Path(__file__).parent / "golden"


def _block_table(cs):
    lib = _native.cuda_lib()
    arr = np.frombuffer(cs, np.uint8)
    count = ctypes.c_size_t()
    elems = ctypes.c_uint64()
    lib.sgn_j2k_ht_block_table(arr.ctypes.data, arr.nbytes, None, 0, ctypes.byref(count), ctypes.byref(elems))
    blocks = (SgnHtBlock * count.value)()
    st = lib.sgn_j2k_ht_block_table(arr.ctypes.data, arr.nbytes, blocks, count.value, ctypes.byref(count),
                                    ctypes.byref(elems))
    assert st == 0, _native.last_error()
    return blocks, count.value, elems.value


def _existing_path_coefficients(cs, fmt):
    """HT-stage output of the regular (allocating) plan path for one tile."""
    plan = Plan([cs], int(fmt))
    plan.execute_async()
    st, _ = plan.wait()
    assert st == 0
    count = ctypes.c_size_t()
    _native.cuda_lib().sgn_plan_tile_coefficients(plan.ctx.handle, plan.handle, 0, None, 0, ctypes.byref(count))
    out = np.zeros(count.value, np.int32)
    st = _native.cuda_lib().sgn_plan_tile_coefficients(plan.ctx.handle, plan.handle, 0, out.ctypes.data, out.size,
                                                       ctypes.byref(count))
    assert st == 0, _native.last_error()
    plan.destroy()
    return out


def _cases():
    fx = json.loads((GOLDEN / "openhtj2k.json").read_text())["fixtures"]["openhtj2k_ds0_ht_12_b11"]
    refine = bytes.fromhex(fx["j2k_hex"])  # carries SigProp/MagRef passes
    rgb = encode.config0().tiles[0].codestream
    return [("refinement_fixture", refine, PixelFormat.Gray8), ("rgb8_256", rgb, PixelFormat.Rgb8)]


@pytest.mark.parametrize("name,cs,fmt", _cases(), ids=[c[0] for c in _cases()])
def test_noalloc_matches_existing_path_on_two_calls(name, cs, fmt):
    import torch

    want = _existing_path_coefficients(cs, fmt)
    blocks, n, elems = _block_table(cs)
    assert elems == want.size
    dev = torch.device("cuda", 0)
    segments = torch.tensor(np.frombuffer(cs, np.uint8).copy(), device=dev)
    coef = torch.empty(elems, dtype=torch.int32, device=dev)
    status = torch.full((1,), 7, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    lib = _native.cuda_lib()
    for call in range(2):
        # Poison the output so a block the call skipped would show up.
        coef.fill_(-123456789)
        st = lib.sgn_ht_decode_blocks_noalloc(blocks, n, segments.data_ptr(), segments.numel(), coef.data_ptr(),
                                              coef.numel(), status.data_ptr(), 1, ctypes.c_void_p(stream.cuda_stream))
        assert st == 0, _native.last_error()
        torch.cuda.synchronize(dev)
        assert int(status.item()) == 0, f"call {call}: block decode failure reported"
        got = coef.cpu().numpy()
        assert np.array_equal(got, want), f"call {call}: coefficients differ from the existing path"


def test_noalloc_clamps_refinement_passes_as_the_parser_does():
    """A descriptor with 29 missing MSBs has one bit-plane left: the kernels
    run its cleanup pass only (as the codestream parser settles it), so it
    decodes exactly as the same descriptor with passes = 1."""
    import torch

    fx = json.loads((GOLDEN / "openhtj2k.json").read_text())["fixtures"]["openhtj2k_ds0_ht_12_b11"]
    cs = bytes.fromhex(fx["j2k_hex"])
    blocks, n, elems = _block_table(cs)
    assert any(b.passes > 1 for b in blocks[:n])
    dev = torch.device("cuda", 0)
    segments = torch.tensor(np.frombuffer(cs, np.uint8).copy(), device=dev)
    lib = _native.cuda_lib()
    outs = []
    for passes in (None, 1):
        tbl = (SgnHtBlock * n)()
        ctypes.memmove(tbl, blocks, ctypes.sizeof(SgnHtBlock) * n)
        for b in tbl:
            if b.passes > 1:
                b.missing_msbs = 29
                if passes is not None:
                    b.passes = passes
        coef = torch.full((elems,), -7, dtype=torch.int32, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        st = lib.sgn_ht_decode_blocks_noalloc(tbl, n, segments.data_ptr(), segments.numel(), coef.data_ptr(),
                                              coef.numel(), status.data_ptr(), 1, None)
        assert st == 0, _native.last_error()
        torch.cuda.synchronize(dev)
        outs.append((coef.cpu().numpy(), int(status.item())))
    assert np.array_equal(outs[0][0], outs[1][0]) and outs[0][1] == outs[1][1]


def test_noalloc_rejects_requests_beyond_its_limit():
    """Every rejection happens on the host, before any device work: too many
    blocks, a block too large, a misaligned coefficient buffer, and blocks
    reaching outside the caller's buffers."""
    lib = _native.cuda_lib()
    blocks = (SgnHtBlock * 4097)()
    st = lib.sgn_ht_decode_blocks_noalloc(blocks, 4097, ctypes.c_void_p(16), 1 << 20, ctypes.c_void_p(16), 1 << 20,
                                          ctypes.c_void_p(16), 1, None)
    assert st == 9  # SGN_ERR_INVALID_ARGUMENT
    assert "4096" in _native.last_error()
    one = (SgnHtBlock * 1)()
    one[0].w, one[0].h, one[0].stride, one[0].passes, one[0].lcup = 128, 64, 128, 1, 10
    st = lib.sgn_ht_decode_blocks_noalloc(one, 1, ctypes.c_void_p(16), 1 << 20, ctypes.c_void_p(16), 1 << 20,
                                          ctypes.c_void_p(16), 1, None)
    assert st == 9
    one[0].w, one[0].h, one[0].stride = 64, 64, 64
    # A coefficient buffer offset by one element (4-byte aligned only).
    st = lib.sgn_ht_decode_blocks_noalloc(one, 1, ctypes.c_void_p(16), 1 << 20, ctypes.c_void_p(20), 1 << 20,
                                          ctypes.c_void_p(16), 1, None)
    assert st == 9 and "aligned" in _native.last_error()
    # The cleanup segment ends past the segment buffer.
    one[0].src = 100
    st = lib.sgn_ht_decode_blocks_noalloc(one, 1, ctypes.c_void_p(16), 109, ctypes.c_void_p(16), 1 << 20,
                                          ctypes.c_void_p(16), 1, None)
    assert st == 2  # SGN_ERR_BUFFER
    # The block's last row ends past the coefficient buffer.
    one[0].src, one[0].dst = 0, 10
    st = lib.sgn_ht_decode_blocks_noalloc(one, 1, ctypes.c_void_p(16), 1 << 20, ctypes.c_void_p(16), 64 * 64 + 9,
                                          ctypes.c_void_p(16), 1, None)
    assert st == 2
