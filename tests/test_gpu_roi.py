"""GPU parity of pruned region decodes: region and region-at-reduced-
resolution requests on large tiles, where only the code blocks and IDWT
windows the region needs are decoded (RoiPlan,
crates/signinum-j2k-native/src/j2c/roi.rs:18-270), must equal the oracle's
region decode (a crop of its full decode, crates/signinum-j2k/tests/decode.rs:374-397)
bit for bit, for reversible HT, irreversible 9/7 and classic code blocks,
gray and RGB, 32x32 and 64x64 blocks, regions anywhere in the tile, alone
and in batches beside full decodes."""
import numpy as np
import pytest

from oracle import oracle
from signinum_b200 import BackendRequest, Codec, Downscale, J2kDecoder, PixelFormat, Rect, encode
from signinum_b200.j2k_cuda import _request

pytestmark = pytest.mark.gpu


def _tiles():
    rgb = encode.he_rgb8(71, 1024, 768, 14.0)
    gray = encode.fluor_gray16(72, 640, 1024)
    return {
        "ht_rgb_64": (encode.encode_lossless(rgb, 1024, 768, 3, 8, levels=6, cb_exp=4), 1024, 768, PixelFormat.Rgb8),
        "ht_rgb_32": (encode.encode_lossless(rgb, 1024, 768, 3, 8, levels=5, cb_exp=3), 1024, 768, PixelFormat.Rgb8),
        "ht_gray16": (encode.encode_lossless(gray, 640, 1024, 1, 16, levels=6, cb_exp=4, use_mct=False), 640, 1024,
                      PixelFormat.Gray16),
        "lossy_rgb": (encode.encode_irreversible(rgb, 1024, 768, 3, 8, 1 / 256, levels=5, cb_exp=4), 1024, 768,
                      PixelFormat.Rgb8),
        "classic_rgb": (encode.encode_classic(rgb[: 512 * 384 * 3], 512, 384, 3, 8, style=0, levels=4, cb_exp=4), 512,
                        384, PixelFormat.Rgb8),
    }


TILES = _tiles()


def _regions(w, h, rng, n):
    out = [Rect(0, 0, 1, 1), Rect(0, 0, 64, 64), Rect(w // 2, h // 3, 64, 64), Rect(w - 65, h - 65, 64, 64),
           Rect(17, h // 2, 255, 3), Rect(w // 3, 5, 1, 200)]
    for _ in range(n):
        rw, rh = int(rng.integers(1, min(300, w))), int(rng.integers(1, min(300, h)))
        out.append(Rect(int(rng.integers(0, w - rw + 1)), int(rng.integers(0, h - rh + 1)), rw, rh))
    return [r for r in out if r.x + r.w <= w and r.y + r.h <= h]


@pytest.mark.parametrize("name", list(TILES))
def test_pruned_regions_match_oracle(name):
    cs, w, h, fmt = TILES[name]
    rng = np.random.default_rng(hash(name) & 0xFFFF)
    dec = J2kDecoder(cs)
    for roi in _regions(w, h, rng, 10):
        got = dec.decode_region_to_device(fmt, roi, BackendRequest.Cuda)
        want, ww, wh = oracle.decode(cs, int(fmt), 1, (roi.x, roi.y, roi.w, roi.h), 1)
        assert got.dimensions() == (ww, wh)
        assert got.to_bytes() == want, (name, roi)
    for scale in (Downscale.Half, Downscale.Quarter):
        d = scale.denominator()
        for roi in _regions(w // d, h // d, rng, 4):
            full = Rect(roi.x * d, roi.y * d, roi.w * d, roi.h * d)
            got = dec.decode_region_scaled_to_device(fmt, full, scale, BackendRequest.Cuda)
            want, ww, wh = oracle.decode(cs, int(fmt), 3, (full.x, full.y, full.w, full.h), d)
            assert got.dimensions() == (ww, wh)
            assert got.to_bytes() == want, (name, full, scale)


def test_pruned_regions_in_a_batch_beside_full_decodes():
    cs, w, h, fmt = TILES["ht_rgb_64"]
    rng = np.random.default_rng(9)
    rois = _regions(w, h, rng, 12)
    inputs, reqs, want = [], [], []
    for k, roi in enumerate(rois):
        inputs.append(cs)
        if k % 3 == 0:
            reqs.append(_request(0))
            want.append(oracle.decode(cs, int(fmt))[0])
        else:
            reqs.append(_request(1, roi))
            want.append(oracle.decode(cs, int(fmt), 1, (roi.x, roi.y, roi.w, roi.h), 1)[0])
    surfaces = Codec.decode_tiles_to_device(inputs, fmt, BackendRequest.Cuda, requests=reqs)
    for s, wnt in zip(surfaces, want):
        assert s.to_bytes() == wnt
