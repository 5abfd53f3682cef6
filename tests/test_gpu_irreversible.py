"""GPU parity of the irreversible path (9/7, dequantisation, ICT) against the
oracle, through the C ABI.

Tolerance: none.  The kernels perform the reference's f32 operations in the
reference's order with explicit rounding (no contracted multiply-adds), so
every output byte must equal the oracle's.
"""
import json
import pathlib

import numpy as np
import pytest

from oracle import oracle
from signinum_b200 import Codec, BackendRequest, Downscale, Error, PixelFormat, Rect, encode
from tests.helpers import random_codestream, random_irreversible
from tests.test_gpu_decode import cpu, gpu

pytestmark = pytest.mark.gpu

GOLDEN = pathlib.Path(__file__).parent / "golden"


def test_golden_irreversible_fixture():
    # OpenJPH-decoded 17x37 gray 9/7 codestream with refinement passes.
    fx = json.loads((GOLDEN / "openhtj2k.json").read_text())["fixtures"]["openhtj2k_ds0_ht_09_b11"]
    got, dims = gpu(bytes.fromhex(fx["j2k_hex"]), PixelFormat.Gray8)
    assert dims == (17, 37)
    assert got == bytes.fromhex(fx["gray_hex"])


@pytest.mark.parametrize("seed", range(6))
def test_random_irreversible_tiles_match_oracle(seed):
    rng = np.random.default_rng(9700 + seed)
    for _ in range(20):
        cs, px, w, h, comps, bd = random_irreversible(rng, max_side=150)
        fmts = [PixelFormat.Rgb8, PixelFormat.Rgba8, PixelFormat.Rgb16] if comps == 3 else \
            [PixelFormat.Gray8, PixelFormat.Gray16]
        for fmt in fmts:
            want, wd = cpu(cs, fmt)
            got, gd = gpu(cs, fmt)
            assert gd == wd == (w, h)
            assert got == want, (w, h, comps, bd, fmt)


@pytest.mark.parametrize("seed", range(2))
def test_irreversible_region_scaled_requests_match_oracle(seed):
    rng = np.random.default_rng(9800 + seed)
    for _ in range(10):
        cs, px, w, h, comps, bd = random_irreversible(rng, max_side=200)
        fmt = PixelFormat.Rgb8 if comps == 3 else PixelFormat.Gray8
        x, y = int(rng.integers(0, w)), int(rng.integers(0, h))
        roi = Rect(x, y, int(rng.integers(0, w - x + 1)), int(rng.integers(0, h - y + 1)))
        for kind, scale in ((1, None), (2, Downscale.Half), (2, Downscale.Quarter), (3, Downscale.Half),
                            (3, Downscale.Eighth)):
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


def test_large_irreversible_rgb_tile():
    px = encode.he_rgb8(31, 1024, 768)
    cs = encode.encode_irreversible(px, 1024, 768, 3, 8, 1 / 512, levels=5)
    got, dims = gpu(cs, PixelFormat.Rgb8)
    assert dims == (1024, 768)
    assert got == cpu(cs, PixelFormat.Rgb8)[0]
    err = np.abs(np.frombuffer(got, np.uint8).astype(int) - px.astype(int))
    assert err.mean() < 2.0


def test_batch_mixing_reversible_and_irreversible_tiles():
    rng = np.random.default_rng(4242)
    tiles = []
    for k in range(16):
        while True:
            cs, _, w, h, comps, _ = (random_irreversible if k % 2 else random_codestream)(rng, max_side=300)
            if comps == 3:
                break
        tiles.append(cs)
    surfaces = Codec.decode_tiles_to_device(tiles, PixelFormat.Rgb8, BackendRequest.Cuda)
    for cs, s in zip(tiles, surfaces):
        want, wd = cpu(cs, PixelFormat.Rgb8)
        assert s.dimensions() == wd
        assert s.to_bytes() == want
