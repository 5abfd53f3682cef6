"""GPU parity: the sm_100a decode path against the oracle, through the C ABI.

Bit-exact on every sample (integer reversible path), plus the adapter
contract of crates/signinum-j2k-cuda/tests/host_surface.rs.
"""
import json
import pathlib

import numpy as np
import pytest

from oracle import oracle
from signinum_b200 import (BackendKind, BackendRequest, Codec, CudaSession, Downscale, Error, J2kDecoder, PixelFormat,
                           Rect, TileBatchError, encode)
from signinum_b200.j2k_cuda import _request
from tests.helpers import WIDE_BLOCKS, precinct_codestream, random_codestream, random_tile, wide_block_codestream

pytestmark = pytest.mark.gpu

GOLDEN = pathlib.Path(__file__).parent / "golden"


def gpu(cs, fmt, kind=0, roi=None, scale=None):
    dec = J2kDecoder(cs)
    if kind == 0:
        s = dec.decode_to_device(fmt, BackendRequest.Cuda)
    elif kind == 1:
        s = dec.decode_region_to_device(fmt, roi, BackendRequest.Cuda)
    elif kind == 2:
        s = dec.decode_scaled_to_device(fmt, scale, BackendRequest.Cuda)
    else:
        s = dec.decode_region_scaled_to_device(fmt, roi, scale, BackendRequest.Cuda)
    return s.to_bytes(), s.dimensions()


def cpu(cs, fmt, kind=0, roi=None, scale=None):
    r = (roi.x, roi.y, roi.w, roi.h) if roi else (0, 0, 0, 0)
    d = scale.denominator() if scale else 1
    got, w, h = oracle.decode(cs, int(fmt), kind, r, d)
    return got, (w, h)


def test_golden_fixture_with_refinement_passes():
    fx = json.loads((GOLDEN / "openhtj2k.json").read_text())["fixtures"]["openhtj2k_ds0_ht_12_b11"]
    got, dims = gpu(bytes.fromhex(fx["j2k_hex"]), PixelFormat.Gray8)
    assert dims == (3, 5)
    assert got == bytes.fromhex(fx["gray_hex"])


def test_config0_tile_bit_exact_and_lossless():
    t = encode.config0(keep_pixels=True).tiles[0]
    got, dims = gpu(t.codestream, PixelFormat.Rgb8)
    assert dims == (256, 256)
    assert got == cpu(t.codestream, PixelFormat.Rgb8)[0]
    assert got == t.pixels.tobytes()


@pytest.mark.parametrize("seed", range(6))
def test_random_tiles_match_oracle(seed):
    rng = np.random.default_rng(77 + seed)
    for _ in range(25):
        cs, px, w, h, comps, bd = random_codestream(rng)
        fmts = [PixelFormat.Rgb8, PixelFormat.Rgba8, PixelFormat.Rgb16] if comps == 3 else \
            [PixelFormat.Gray8, PixelFormat.Gray16]
        for fmt in fmts:
            want, wd = cpu(cs, fmt)
            got, gd = gpu(cs, fmt)
            assert gd == wd == (w, h)
            assert got == want, (w, h, comps, bd, fmt)


@pytest.mark.parametrize("cb", WIDE_BLOCKS)
def test_wide_code_blocks_match_oracle(cb):
    """Blocks wider than 64 take the kernels' wide paths (VLC context read
    back from the symbol table, MagSgn exponents kept per column in shared
    memory); 4x1024 blocks the long narrow ones."""
    rng = np.random.default_rng(4100 + 16 * cb[0] + cb[1])
    for _ in range(3):
        cs, px, w, h, comps, bd = wide_block_codestream(rng, cb)
        fmts = [PixelFormat.Rgb8, PixelFormat.Rgb16] if comps == 3 else [PixelFormat.Gray8, PixelFormat.Gray16]
        for fmt in fmts:
            want, wd = cpu(cs, fmt)
            got, gd = gpu(cs, fmt)
            assert gd == wd == (w, h)
            assert got == want, (cb, w, h, comps, bd, fmt)
        roi = Rect(w // 5, h // 4, max(1, w // 2), max(1, h // 2))
        fmt = fmts[0]
        assert gpu(cs, fmt, 1, roi)[0] == cpu(cs, fmt, 1, roi)[0]


@pytest.mark.parametrize("kind", ["ht", "classic", "lossy"])
def test_precinct_partitions_match_oracle(kind):
    """Codestreams cut into precincts (2 .. 256 samples a side) in every
    progression, over several tile-parts: HT, multi-layer classic and lossy
    9/7 code blocks."""
    rng = np.random.default_rng({"ht": 4500, "classic": 4501, "lossy": 4502}[kind])
    for _ in range(12):
        cs, px, w, h, comps = precinct_codestream(rng, kind)
        fmt = PixelFormat.Rgb8 if comps == 3 else PixelFormat.Gray8
        want, wd = cpu(cs, fmt)
        got, gd = gpu(cs, fmt)
        assert gd == wd == (w, h)
        assert got == want, (kind, w, h, comps)
        if kind != "lossy":
            assert got == px.tobytes()


@pytest.mark.parametrize("seed", range(3))
def test_region_scaled_requests_match_oracle(seed):
    rng = np.random.default_rng(500 + seed)
    for _ in range(12):
        cs, px, w, h, comps, bd = random_codestream(rng, max_side=140)
        fmt = PixelFormat.Rgb8 if comps == 3 else PixelFormat.Gray8
        x, y = int(rng.integers(0, w)), int(rng.integers(0, h))
        roi = Rect(x, y, int(rng.integers(0, w - x + 1)), int(rng.integers(0, h - y + 1)))
        for kind, scale in ((1, None), (2, Downscale.Half), (2, Downscale.Quarter), (3, Downscale.Half),
                            (3, Downscale.Quarter), (3, Downscale.Eighth)):
            try:
                want = cpu(cs, fmt, kind, roi, scale)
            except oracle.OracleError as e:
                with pytest.raises(Error) as g:
                    gpu(cs, fmt, kind, roi, scale)
                assert g.value.status == e.status
                continue
            got = gpu(cs, fmt, kind, roi, scale)
            assert got[1] == want[1]
            assert got[0] == want[0], (w, h, comps, bd, kind, roi, scale)


def test_batch_preserves_order_and_matches_single_decodes():
    w = encode.config2(n=24)
    tiles = [t.codestream for t in w.tiles]
    surfaces = Codec.decode_tiles_to_device(tiles, PixelFormat.Rgb8, BackendRequest.Cuda)
    assert len(surfaces) == len(tiles)
    for t, s in zip(w.tiles, surfaces):
        assert s.dimensions() == (t.width, t.height)
        assert s.to_bytes() == cpu(t.codestream, PixelFormat.Rgb8)[0]


def test_batch_reports_lowest_failing_index():
    w = encode.config2(n=6)
    tiles = [t.codestream for t in w.tiles]
    bad = bytearray(tiles[4])
    tiles[4] = bytes(bad[:40])  # truncated inside the main header
    tiles[2] = b"\x00\x01not a codestream"
    with pytest.raises(TileBatchError) as e:
        Codec.decode_tiles_to_device(tiles, PixelFormat.Rgb8, BackendRequest.Cuda)
    assert e.value.index == 2


def test_corrupt_code_block_is_an_error_not_a_fault():
    t = encode.config0().tiles[0]
    cs = bytearray(t.codestream)
    # Flip bytes inside the packet bodies (after the main header).
    rng = np.random.default_rng(3)
    for pos in rng.integers(len(cs) // 2, len(cs) - 2, 64):
        cs[pos] ^= 0xA5
    try:
        got, _ = gpu(bytes(cs), PixelFormat.Rgb8)
    except Error as e:
        assert e.status in (3, 4)
        try:
            cpu(bytes(cs), PixelFormat.Rgb8)
        except oracle.OracleError:
            pass
    else:
        # When the oracle also decodes the damaged stream the bytes must agree.
        try:
            want = cpu(bytes(cs), PixelFormat.Rgb8)[0]
        except oracle.OracleError:
            return
        assert got == want


@pytest.mark.parametrize("seed", range(2))
@pytest.mark.parametrize("where", ["magsgn", "vlc"])
@pytest.mark.parametrize("form", [0, 1])
def test_damaged_narrow_blocks_stay_in_their_tile(seed, where, form):
    """Code blocks at most 32 wide decode two per warp in the two-pass form
    (form 0), and the two may come from different tiles of the batch; the
    fused form (1) decodes each in a CTA whose MagSgn warp waits on the
    block's chain row by row.  Damage in a tile's MagSgn bits must give the
    oracle's (different) values; damage in its VLC bits must fail that tile
    alone; the tiles decoded beside it must come out exact."""
    from signinum_b200.plan import Plan

    rng = np.random.default_rng(4700 + seed)
    pixels, inputs = [], []
    for _ in range(5):
        px = random_tile(rng, 96, 80, 3, 8, 1)
        pixels.append(px)
        inputs.append(encode.encode_lossless(px.reshape(-1), 96, 80, 3, 8, levels=2, cb_exp=3))
    # Damage the cleanup segments of some of tile 2's coded blocks (packet
    # headers intact): near the start (MagSgn bits) or near the end (VLC).
    import ctypes

    from signinum_b200 import _native
    from signinum_b200._native import SgnHtBlock

    lib = _native.cuda_lib()
    arr = np.frombuffer(inputs[2], np.uint8)
    count, elems = ctypes.c_size_t(), ctypes.c_size_t()
    lib.sgn_j2k_ht_block_table(arr.ctypes.data, arr.nbytes, None, 0, ctypes.byref(count), ctypes.byref(elems))
    blocks = (SgnHtBlock * count.value)()
    assert lib.sgn_j2k_ht_block_table(arr.ctypes.data, arr.nbytes, blocks, count.value, ctypes.byref(count),
                                      ctypes.byref(elems)) == 0
    coded = [b for b in blocks if b.passes == 1 and b.lcup >= 16 and b.w <= 32]
    assert coded
    cs = bytearray(inputs[2])
    for b in coded[:: max(1, len(coded) // 8)]:
        cs[b.src + (1 if where == "magsgn" else b.lcup - 4)] ^= 0x5A
    inputs[2] = bytes(cs)
    plan = Plan(inputs, PixelFormat.Rgb8)
    plan.set_cleanup_form(form)
    plan.execute_async()
    _, per = plan.wait()
    for i in (0, 1, 3, 4):
        assert per[i] == 0
        assert plan.download(i) == pixels[i].tobytes()
    if where == "magsgn":
        want = cpu(inputs[2], PixelFormat.Rgb8)[0]
        assert want != pixels[2].tobytes()
        assert per[2] == 0
        assert plan.download(2) == want
    else:
        with pytest.raises(oracle.OracleError):
            cpu(inputs[2], PixelFormat.Rgb8)
        assert per[2] in (3, 4)
    plan.destroy()


def test_unsupported_format_rejected_before_device_work():
    # host_surface.rs:59-68
    t = encode.config0().tiles[0]
    with pytest.raises(Error) as e:
        J2kDecoder(t.codestream).decode_to_device(PixelFormat.Rgba16, BackendRequest.Cuda)
    assert e.value.is_unsupported()


def test_invalid_region_rejected():
    t = encode.config0().tiles[0]
    with pytest.raises(Error) as e:
        J2kDecoder(t.codestream).decode_region_to_device(PixelFormat.Rgb8, Rect(200, 0, 100, 10),
                                                         BackendRequest.Cuda)
    assert e.value.is_invalid_region()


def test_cuda_surface_contract_and_padded_download():
    # host_surface.rs:71-98, :144-172
    t = encode.config0(keep_pixels=True).tiles[0]
    s = J2kDecoder(t.codestream).decode_to_device(PixelFormat.Rgb8, BackendRequest.Cuda)
    assert s.backend_kind() == BackendKind.Cuda
    assert s.as_host_bytes() is None
    assert s.cuda_surface().device_ptr() != 0
    assert s.cuda_surface().stats().kernel_dispatches() > 0
    assert s.pitch_bytes() == 256 * 3 and s.byte_len() == 256 * 256 * 3
    stride = 256 * 3 + 13
    out = np.zeros(stride * 256, np.uint8)
    s.download_into(out, stride)
    rows = out.reshape(256, stride)[:, : 256 * 3]
    assert rows.tobytes() == t.pixels.tobytes()
    with pytest.raises(Error) as e:
        s.download_into(np.zeros(10, np.uint8), stride)
    assert e.value.is_buffer_error()


def test_session_reuse_counts_submissions():
    # host_surface.rs:225-268
    t = encode.config0().tiles[0]
    session = CudaSession()
    assert not session.is_runtime_initialized()
    dec = J2kDecoder(t.codestream)
    a = dec.decode_to_device(PixelFormat.Rgb8, BackendRequest.Cuda, session)
    b = dec.decode_to_device(PixelFormat.Rgb8, BackendRequest.Cuda, session)
    assert session.submissions() == 2 and session.is_runtime_initialized()
    assert a.to_bytes() == b.to_bytes()


def test_gray16_and_high_bit_depth_tiles():
    px = encode.fluor_gray16(9, 256, 192)
    cs = encode.encode_lossless(px, 256, 192, 1, 16, levels=6, cb_exp=4, use_mct=False)
    got, dims = gpu(cs, PixelFormat.Gray16)
    assert dims == (256, 192)
    assert got == px.tobytes()
    for fmt in (PixelFormat.Gray8,):
        assert gpu(cs, fmt)[0] == cpu(cs, fmt)[0]
        roi = Rect(5, 7, 100, 50)
        assert gpu(cs, fmt, 1, roi)[0] == cpu(cs, fmt, 1, roi)[0]
