"""GPU parity of classic (EBCOT Tier-1) code-block decoding against the
oracle, through the C ABI: every code-block style, lossless and lossy, all
pixel formats, regions and reduced resolutions, and batches mixing HT and
classic tiles.  Tolerance: none (the MQ decoder and the passes are integer
arithmetic; the 9/7 stages are the irreversible path's exact f32)."""
import numpy as np
import pytest

from oracle import oracle
from signinum_b200 import BackendRequest, Codec, Downscale, Error, PixelFormat, Rect, encode
from tests.helpers import CLASSIC_STYLES, random_classic, random_codestream
from tests.test_gpu_decode import cpu, gpu

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", range(5))
def test_random_classic_tiles_match_oracle(seed):
    rng = np.random.default_rng(5100 + seed)
    for _ in range(16):
        cs, px, w, h, comps, bd = random_classic(rng, max_side=140)
        fmts = [PixelFormat.Rgb8, PixelFormat.Rgba8, PixelFormat.Rgb16] if comps == 3 else \
            [PixelFormat.Gray8, PixelFormat.Gray16]
        for fmt in fmts:
            want, wd = cpu(cs, fmt)
            got, gd = gpu(cs, fmt)
            assert gd == wd == (w, h)
            assert got == want, (w, h, comps, bd, fmt)


@pytest.mark.parametrize("style", CLASSIC_STYLES)
def test_classic_styles_on_a_full_tile(style):
    px = encode.he_rgb8(11 + style, 512, 512)
    cs = encode.encode_classic(px, 512, 512, 3, 8, style=style, levels=5)
    got, dims = gpu(cs, PixelFormat.Rgb8)
    assert dims == (512, 512)
    assert got == px.tobytes()  # lossless
    assert got == cpu(cs, PixelFormat.Rgb8)[0]


def test_classic_region_and_scaled_requests_match_oracle():
    rng = np.random.default_rng(5200)
    for _ in range(10):
        cs, px, w, h, comps, bd = random_classic(rng, max_side=200)
        fmt = PixelFormat.Rgb8 if comps == 3 else PixelFormat.Gray8
        x, y = int(rng.integers(0, w)), int(rng.integers(0, h))
        roi = Rect(x, y, int(rng.integers(0, w - x + 1)), int(rng.integers(0, h - y + 1)))
        for kind, scale in ((1, None), (2, Downscale.Half), (3, Downscale.Quarter)):
            try:
                want = cpu(cs, fmt, kind, roi, scale)
            except oracle.OracleError as e:
                with pytest.raises(Error) as g:
                    gpu(cs, fmt, kind, roi, scale)
                assert g.value.status == e.status
                continue
            got = gpu(cs, fmt, kind, roi, scale)
            assert got == want, (w, h, comps, bd, kind, roi, scale)


def test_batch_mixing_ht_and_classic_tiles():
    rng = np.random.default_rng(5300)
    tiles = []
    while len(tiles) < 16:
        cs, _, w, h, comps, _ = (random_classic if len(tiles) % 2 else random_codestream)(rng, max_side=300)
        if comps == 3:
            tiles.append(cs)
    surfaces = Codec.decode_tiles_to_device(tiles, PixelFormat.Rgb8, BackendRequest.Cuda)
    for cs, s in zip(tiles, surfaces):
        want, wd = cpu(cs, PixelFormat.Rgb8)
        assert s.dimensions() == wd
        assert s.to_bytes() == want


@pytest.mark.parametrize("layers", [2, 5])
def test_multi_layer_classic_tiles(layers):
    # Quality layers: the host gathers each block's parts from all packets.
    for style, prog in ((0, 0), (0x01, 1), (0x04, 2), (0x2F, 3), (0x05, 4)):
        px = encode.he_rgb8(21 + style, 384, 256)
        cs = encode.encode_classic(px, 384, 256, 3, 8, style=style, levels=4, progression=prog, layers=layers)
        got, dims = gpu(cs, PixelFormat.Rgb8)
        assert dims == (384, 256)
        assert got == px.tobytes()
        assert got == cpu(cs, PixelFormat.Rgb8)[0]
