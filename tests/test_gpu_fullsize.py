"""GPU parity at the benchmark workloads' full sizes.

Every tile of the uniform batch (256 x 512^2 RGB8), the uneven batch (1024
tiles, sides 128..1024) and the high-bit-depth batch (128 x 2048^2 u16 gray,
6 levels) decodes bit-exactly against the oracle (the restated reference CPU
tile batch, crates/signinum-j2k/src/batch.rs:110-147) and against the source
pixels (lossless identity, crates/signinum-j2k/src/encode.rs:459-502),
through the batched plan, the batched drop-in call and, on a spread of
tiles, the plain per-tile call; and over a thousand mixed serving requests
each equal the oracle's decode of that request.  The tolerance is zero: the
reversible path is integer arithmetic.
"""
import os

import numpy as np
import pytest

from oracle import oracle
from signinum_b200 import BackendRequest, Codec, Downscale, J2kDecoder, PixelFormat, Rect, encode
from signinum_b200.plan import Plan
from signinum_b200.server import Server, collect

pytestmark = pytest.mark.gpu

CORES = os.cpu_count() or 1


def _oracle_chunks(tiles, fmt, chunk=64):
    """(index, oracle bytes) of every tile, decoded in chunks on all cores."""
    for s in range(0, len(tiles), chunk):
        outs, first = oracle.decode_batch([t.codestream for t in tiles[s:s + chunk]], int(fmt), workers=CORES)
        assert first == -1
        for k, o in enumerate(outs):
            t = tiles[s + k]
            yield s + k, o[: t.width * t.height * (3 if fmt == PixelFormat.Rgb8 else 2)].tobytes()


def test_uniform_batch_every_tile_bit_exact():
    """256 tiles of 512x512 RGB8: all through one batched plan (the graph
    replay of its second execution), a spread of 16 through the plain call."""
    w = encode.config1(keep_pixels=True)
    tiles = w.tiles
    plan = Plan([t.codestream for t in tiles], int(PixelFormat.Rgb8))
    plan.execute_async()
    plan.execute_async()  # the second execution replays the captured graph
    st, per = plan.wait()
    assert st == 0 and all(p == 0 for p in per)
    for i, want in _oracle_chunks(tiles, PixelFormat.Rgb8):
        got = plan.download(i)
        assert got == want, f"tile {i} differs from the oracle"
        assert got == tiles[i].pixels.tobytes(), f"tile {i} is not lossless"
    plan.destroy()
    for i in range(0, len(tiles), 16):
        s = J2kDecoder(tiles[i].codestream).decode_to_device(PixelFormat.Rgb8, BackendRequest.Cuda)
        assert s.to_bytes() == tiles[i].pixels.tobytes(), f"plain call, tile {i}"


def test_uneven_batch_every_tile_bit_exact():
    """The 1024 uneven tiles through the batched drop-in call
    (decode_tiles_to_device: chunked upload / parse / decode pipeline) and
    through one device-resident plan."""
    w = encode.config2(keep_pixels=True)
    tiles = w.tiles
    assert len(tiles) == 1024
    surfaces = Codec.decode_tiles_to_device([t.codestream for t in tiles], PixelFormat.Rgb8, BackendRequest.Cuda)
    plan = Plan([t.codestream for t in tiles], int(PixelFormat.Rgb8))
    plan.execute_async()
    st, _ = plan.wait()
    assert st == 0
    for i, want in _oracle_chunks(tiles, PixelFormat.Rgb8):
        assert surfaces[i].dimensions() == (tiles[i].width, tiles[i].height)
        got = surfaces[i].to_bytes()
        assert got == want, f"tile {i} ({tiles[i].width}x{tiles[i].height}, {tiles[i].kind}) differs from the oracle"
        assert got == tiles[i].pixels.tobytes(), f"tile {i} is not lossless"
        assert plan.download(i) == want, f"plan, tile {i}"
        surfaces[i].free()
    plan.destroy()


def test_high_bit_depth_batch_every_tile_bit_exact():
    """128 gray u16 tiles of 2048x2048 (6 levels, 1,027 code blocks each):
    Gray16 output of one batched plan, every sample, against the oracle and
    the source; Gray8 of a spread against the oracle."""
    w = encode.config3()
    tiles = w.tiles
    plan = Plan([t.codestream for t in tiles], int(PixelFormat.Gray16))
    plan.execute_async()
    plan.execute_async()
    st, per = plan.wait()
    assert st == 0 and all(p == 0 for p in per)
    for i, want in _oracle_chunks(tiles, PixelFormat.Gray16, chunk=16):
        got = plan.download(i)
        assert got == want, f"tile {i} differs from the oracle"
        src = encode.fluor_gray16(encode._mix(encode.MASTER_SEED, 3, i), 2048, 2048)
        assert got == src.tobytes(), f"tile {i} is not lossless"
    plan.destroy()
    for i in range(0, len(tiles), 32):
        s = J2kDecoder(tiles[i].codestream).decode_to_device(PixelFormat.Gray8, BackendRequest.Cuda)
        assert s.to_bytes() == oracle.decode(tiles[i].codestream, int(PixelFormat.Gray8))[0], f"gray8 tile {i}"


def test_serving_thousand_mixed_requests_bit_exact():
    """1,200 requests (60% full RGB8, 25% quarter resolution, 15% 256x256
    region at random offsets) over a pool of uneven tiles, submitted as one
    burst and batched continuously; every result equals the oracle's decode
    of the same request."""
    pool = encode.config4_pool(256).tiles
    rng = np.random.default_rng(0xC4)
    reqs = []
    for _ in range(1200):
        i = int(rng.integers(len(pool)))
        t = pool[i]
        u = rng.uniform()
        if u < 0.6:
            reqs.append((i, None, None))
        elif u < 0.85:
            reqs.append((i, None, Downscale.Quarter))
        else:
            side = min(256, t.width)
            reqs.append((i, Rect(int(rng.integers(0, t.width - side + 1)), int(rng.integers(0, t.height - side + 1)),
                                 side, side), None))
    with Server(device_budget_bytes=16 << 30, resident_capacity_bytes=sum(len(t.codestream) for t in pool) + (1 << 24),
                max_batch_tiles=128, slots=4, max_batch_samples=96_000_000) as srv:
        ids = [srv.register(t.codestream) for t in pool]
        tickets = [srv.submit(ids[i], PixelFormat.Rgb8, roi, scale) for i, roi, scale in reqs]
        got = collect(srv, tickets, timeout_s=120.0)
        batches = {got[t].batch_tiles for t in tickets}
        assert max(batches) > 1, "requests were not batched"
        for t, (i, roi, scale) in zip(tickets, reqs):
            r = got[t]
            assert r.status == 0
            kind = 0 if roi is None and scale is None else 1 if scale is None else 2
            rr = (roi.x, roi.y, roi.w, roi.h) if roi else (0, 0, 0, 0)
            want, ww, wh = oracle.decode(pool[i].codestream, int(PixelFormat.Rgb8), kind, rr,
                                         scale.denominator() if scale else 1)
            assert r.surface.dimensions() == (ww, wh)
            assert r.surface.to_bytes() == want, (i, roi, scale)
            r.surface.free()
