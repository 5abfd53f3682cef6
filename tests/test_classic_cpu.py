"""Classic (EBCOT Tier-1) decoding on the CPU: the oracle's and the product's
context and probability tables pinned to the reference's, and lossless round
trips of the classic encoder through the oracle in every code-block style
(CPU only)."""
import hashlib
import json
import pathlib

import numpy as np
import pytest

from oracle import oracle
from signinum_b200 import encode

GOLDEN = pathlib.Path(__file__).parent / "golden"
STYLES = [0, 0x01, 0x02, 0x04, 0x08, 0x20, 0x05, 0x0D, 0x2F]


def _sha(b):
    return hashlib.sha256(bytes(b)).hexdigest()


def _check(tables, ref):
    zl, zh, zhh, lab, xr, qe = tables
    assert _sha(zl) == ref["ZERO_CTX_LL_LH_LOOKUP"]["sha256"]
    assert _sha(zh) == ref["ZERO_CTX_HL_LOOKUP"]["sha256"]
    assert _sha(zhh) == ref["ZERO_CTX_HH_LOOKUP"]["sha256"]
    assert _sha(lab) == ref["SIGN_CONTEXT_LOOKUP"]["label_sha256"]
    assert _sha(xr) == ref["SIGN_CONTEXT_LOOKUP"]["xor_sha256"]
    assert _sha(qe) == ref["QE_TABLE"]["sha256"]


def test_oracle_ebcot_tables_match_reference():
    _check(oracle.ebcot_tables(), json.loads((GOLDEN / "ebcot_tables_sha256.json").read_text()))


def test_product_ebcot_tables_match_reference():
    from signinum_b200 import _native

    bufs = [np.zeros(256, np.uint8) for _ in range(5)] + [np.zeros(235, np.uint8)]
    _native.cuda_lib().sgn_ebcot_tables(*[b.ctypes.data for b in bufs])
    _check(bufs, json.loads((GOLDEN / "ebcot_tables_sha256.json").read_text()))


@pytest.mark.parametrize("style", STYLES)
def test_classic_round_trip_through_oracle(style):
    # The reference pins its classic decoder the same way: encode, decode,
    # compare (crates/signinum-j2k-native/src/j2c/bitplane.rs:1468-1686).
    rng = np.random.default_rng(1000 + style)
    for w, h, c, bd, levels in [(64, 48, 3, 8, 3), (37, 29, 1, 8, 2), (130, 70, 3, 8, 5), (33, 65, 1, 12, 3),
                                (1, 7, 1, 8, 2), (9, 1, 3, 8, 2), (70, 70, 1, 16, 4)]:
        dt = np.uint8 if bd <= 8 else np.dtype("<u2")
        px = rng.integers(0, 1 << bd, size=w * h * c).astype(dt)
        cs = encode.encode_classic(px.view(np.uint8), w, h, c, bd, style=style, levels=levels)
        fmt = 1 if c == 3 else (3 if bd > 8 else 0)
        got, gw, gh = oracle.decode(cs, fmt)
        assert (gw, gh) == (w, h)
        assert got == px.tobytes(), (style, w, h, c, bd)


@pytest.mark.parametrize("layers", [2, 3, 5])
def test_multi_layer_classic_round_trip_through_oracle(layers):
    # Quality layers: a block's passes split over several packets, its
    # codeword segments continued across them (segment.rs:168-302).
    rng = np.random.default_rng(2000 + layers)
    for style in (0, 0x01, 0x04, 0x05, 0x2F):
        for prog in range(5):
            px = rng.integers(0, 256, size=70 * 50 * 3).astype(np.uint8)
            cs = encode.encode_classic(px, 70, 50, 3, 8, style=style, levels=3, cb_exp=3, progression=prog,
                                       layers=layers)
            assert oracle.decode(cs, 1)[0] == px.tobytes(), (style, prog)


def test_lossy_classic_decodes_like_lossy_ht():
    # Same quantised coefficients, two block coders: the same pixels.
    px = encode.he_rgb8(7, 96, 80)
    b = oracle.decode(encode.encode_irreversible(px, 96, 80, 3, 8, 1 / 512, levels=4), 1)[0]
    for style in (0, 0x05, 0x2F):
        a = encode.encode_classic(px, 96, 80, 3, 8, style=style, irreversible=True, relative_step=1 / 512, levels=4)
        assert oracle.decode(a, 1)[0] == b
