"""GPU tests of the serving loop (sgn_server_*): continuous batching must not
change any result, admission must respect the device-memory budget, and
request validation matches the plain call's."""
import numpy as np
import pytest

from oracle import oracle
from signinum_b200 import Downscale, Error, PixelFormat, Rect, encode
from signinum_b200.server import Server, collect

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pool():
    # Twelve uneven tiles drawn like the uneven batch (sides 128..1024,
    # 32x32/64x64 blocks, near-blank tiles among them).
    return encode.config2(n=12).tiles


def _requests(tiles, n, seed):
    """A mix of full, quarter-resolution and 256x256 region requests."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        i = int(rng.integers(len(tiles)))
        t = tiles[i]
        u = rng.uniform()
        if u < 0.6:
            out.append((i, None, None))
        elif u < 0.85:
            out.append((i, None, Downscale.Quarter))
        else:
            side = min(256, t.width)
            x = int(rng.integers(0, t.width - side + 1))
            y = int(rng.integers(0, t.height - side + 1))
            out.append((i, Rect(x, y, side, side), None))
    return out


def _oracle(t, roi, scale):
    kind = 0 if roi is None and scale is None else 1 if scale is None else 2
    r = (roi.x, roi.y, roi.w, roi.h) if roi else (0, 0, 0, 0)
    d = scale.denominator() if scale else 1
    return oracle.decode(t.codestream, int(PixelFormat.Rgb8), kind, r, d)


def _run(server, ids, reqs):
    tickets = [server.submit(ids[i], PixelFormat.Rgb8, roi, scale) for i, roi, scale in reqs]
    got = collect(server, tickets)
    out = []
    for t in tickets:
        r = got[t]
        assert r.status == 0, r.status
        out.append((r.surface.to_bytes(), r.surface.dimensions(), r))
        r.surface.free()
    return out


def test_results_are_the_same_alone_and_in_the_mix(pool):
    with Server(max_batch_tiles=16, slots=3) as server:
        ids = [server.register(t.codestream) for t in pool]
        mix = _requests(pool, 80, seed=7)
        probes = mix[::9]
        # Alone: one request at a time, each its own batch.
        alone = [_run(server, ids, [q])[0] for q in probes]
        for (i, roi, scale), (b, dims, r) in zip(probes, alone):
            assert r.batch_tiles == 1
            want, w, h = _oracle(pool[i], roi, scale)
            assert dims == (w, h) and b == want
        # In the mix: everything submitted at once, batched and overlapped.
        mixed = _run(server, ids, mix)
        assert max(r.batch_tiles for _, _, r in mixed) > 1
        for q, (b, dims, _) in zip(probes, mixed[::9]):
            assert (b, dims) == alone[probes.index(q)][:2]
        for (i, roi, scale), (b, dims, _) in zip(mix, mixed):
            want, w, h = _oracle(pool[i], roi, scale)
            assert dims == (w, h) and b == want
        st = server.stats()
        assert st["completed"] == len(mix) + len(probes) and st["bytes_in_use"] == 0


def test_admission_keeps_in_flight_batches_within_the_budget(pool):
    big = max(pool, key=lambda t: t.width * t.height)
    # Room for about two of the largest tiles at a time.
    budget = 2 * big.width * big.height * 3 * 8 + (1 << 20)
    with Server(device_budget_bytes=budget, max_batch_tiles=64, slots=4) as server:
        ids = [server.register(t.codestream) for t in pool]
        reqs = [(i, None, None) for i in range(len(pool))] * 3
        res = _run(server, ids, reqs)
        st = server.stats()
        assert st["completed"] == len(reqs)
        assert st["peak_bytes_in_use"] <= budget
        assert st["batches"] > 1
        for (i, _, _), (b, _, _) in zip(reqs, res):
            assert b == _oracle(pool[i], None, None)[0]


def test_submit_validation(pool):
    t = pool[0]
    with Server(device_budget_bytes=1 << 20) as server:
        tid = server.register(t.codestream)
        with pytest.raises(Error) as e:
            server.submit(tid, PixelFormat.Rgb8)  # larger than the whole budget
        assert e.value.status == 10
    with Server() as server:
        tid = server.register(t.codestream)
        with pytest.raises(Error) as e:
            server.submit(tid, PixelFormat.Rgb8, Rect(t.width - 8, 0, 16, 16))
        assert e.value.is_invalid_region()
        with pytest.raises(Error) as e:
            server.submit(tid, PixelFormat.Rgba16)
        assert e.value.is_unsupported()
        with pytest.raises(Error):
            server.submit(tid + 5, PixelFormat.Rgb8)


def test_serving_mixes_ht_lossy_and_classic_tiles():
    # The serving loop batches whatever is registered: HT lossless, lossy 9/7
    # and classic (multi-layer) tiles side by side, each exact.
    px = [encode.he_rgb8(40 + k, 256, 192) for k in range(3)]
    tiles = [encode.encode_lossless(px[0], 256, 192, 3, 8, levels=4),
             encode.encode_irreversible(px[1], 256, 192, 3, 8, 1 / 256, levels=4),
             encode.encode_classic(px[2], 256, 192, 3, 8, style=0x05, levels=4, layers=3)]

    class T:
        def __init__(self, cs):
            self.codestream, self.width, self.height = cs, 256, 192

    pool = [T(cs) for cs in tiles]
    with Server(max_batch_tiles=8, slots=2) as server:
        ids = [server.register(t.codestream) for t in pool]
        reqs = [(i, None, None) for i in range(3)] * 3 + [(2, Rect(32, 16, 128, 96), None), (1, None, Downscale.Half)]
        for (i, roi, scale), (b, dims, _) in zip(reqs, _run(server, ids, reqs)):
            want, w, h = _oracle(pool[i], roi, scale)
            assert dims == (w, h) and b == want
