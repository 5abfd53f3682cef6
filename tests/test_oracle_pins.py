"""The oracle pinned to the reference: golden vectors, lookup tables and
lossless identity (CPU only)."""
import hashlib
import json
import pathlib
import struct

import numpy as np
import pytest

from oracle import oracle
from signinum_b200 import encode
from tests.helpers import WIDE_BLOCKS, precinct_codestream, random_codestream, wide_block_codestream

GOLDEN = pathlib.Path(__file__).parent / "golden"


def _fixtures():
    return json.loads((GOLDEN / "openhtj2k.json").read_text())["fixtures"]


def test_openhtj2k_ds0_ht_12_known_answer():
    # crates/signinum-j2k-native/src/lib.rs:2933-2939: reversible 5/3 with
    # SigProp + MagRef refinement passes, 3x5 gray, decoded samples by OpenJPH.
    fx = _fixtures()["openhtj2k_ds0_ht_12_b11"]
    got, w, h = oracle.decode(bytes.fromhex(fx["j2k_hex"]), 0)
    assert (w, h) == (3, 5)
    assert got == bytes.fromhex(fx["gray_hex"])


def test_openhtj2k_ds0_ht_09_known_answer():
    # crates/signinum-j2k-native/src/lib.rs:2941-2947,3474-3481: irreversible
    # 9/7 with scalar-expounded quantisation, 17x37 gray, decoded samples by
    # OpenJPH.  Exact: the oracle's float lifting rounds the same way here.
    fx = _fixtures()["openhtj2k_ds0_ht_09_b11"]
    got, w, h = oracle.decode(bytes.fromhex(fx["j2k_hex"]), 0)
    assert (w, h) == (17, 37)
    assert got == bytes.fromhex(fx["gray_hex"])


def _sha(arr):
    return hashlib.sha256(struct.pack("<%dH" % len(arr), *[int(v) for v in arr])).hexdigest()


def test_oracle_lookup_tables_match_reference():
    ref = json.loads((GOLDEN / "ht_lookup_sha256.json").read_text())
    for name, arr in zip(("VLC_TABLE0", "VLC_TABLE1", "UVLC_TABLE0", "UVLC_TABLE1"), oracle.tables()):
        assert len(arr) == ref[name]["len"]
        assert _sha(arr) == ref[name]["sha256"], name


def test_product_lookup_tables_match_reference():
    from signinum_b200 import _native

    ref = json.loads((GOLDEN / "ht_lookup_sha256.json").read_text())
    bufs = [np.zeros(n, np.uint16) for n in (1024, 1024, 320, 256)]
    _native.cuda_lib().sgn_ht_lookup_tables(*[b.ctypes.data for b in bufs])
    for name, arr in zip(("VLC_TABLE0", "VLC_TABLE1", "UVLC_TABLE0", "UVLC_TABLE1"), bufs):
        assert _sha(arr) == ref[name]["sha256"], name


@pytest.mark.parametrize("seed", range(4))
def test_encoder_roundtrip_through_oracle(seed):
    rng = np.random.default_rng(1000 + seed)
    for _ in range(40):
        cs, px, w, h, comps, bd = random_codestream(rng)
        fmt = (1 if comps == 3 else 0) if bd == 8 else (4 if comps == 3 else 3)
        got, ow, oh = oracle.decode(cs, fmt)
        assert (ow, oh) == (w, h)
        want = px.tobytes() if bd == 8 or bd == 16 else px.astype("<u2").tobytes()
        if bd not in (8, 16):
            want = np.clip(px.astype(np.int64), 0, (1 << bd) - 1).astype("<u2").tobytes()
        assert got == want


@pytest.mark.parametrize("cb", WIDE_BLOCKS)
def test_wide_code_blocks_roundtrip_through_oracle(cb):
    """Code blocks wider or higher than 64 (up to 1024x4 and 4x1024) decode
    losslessly: the oracle's HT decoder has no 64-sample limit."""
    rng = np.random.default_rng(4000 + 16 * cb[0] + cb[1])
    for _ in range(3):
        cs, px, w, h, comps, bd = wide_block_codestream(rng, cb)
        fmt = (1 if comps == 3 else 0) if bd == 8 else (4 if comps == 3 else 3)
        got, ow, oh = oracle.decode(cs, fmt)
        assert (ow, oh) == (w, h)
        assert got == px.tobytes()


@pytest.mark.parametrize("kind", ["ht", "classic"])
def test_precinct_partitions_roundtrip_through_oracle(kind):
    """Resolutions cut into precincts (code blocks clipped to them, packets
    per precinct in every progression, the position-driven ones included,
    split over tile-parts) decode losslessly: the encoder's packet order and
    the oracle's agree."""
    rng = np.random.default_rng({"ht": 4300, "classic": 4301}[kind])
    for _ in range(30):
        cs, px, w, h, comps = precinct_codestream(rng, kind)
        got, ow, oh = oracle.decode(cs, 1 if comps == 3 else 0)
        assert (ow, oh) == (w, h)
        assert got == px.tobytes()


def test_workload_tile_is_lossless():
    w = encode.config0(keep_pixels=True)
    t = w.tiles[0]
    got, ow, oh = oracle.decode(t.codestream, 1)
    assert (ow, oh) == (256, 256)
    assert got == t.pixels.tobytes()


def test_region_is_crop_of_full_decode():
    # crates/signinum-j2k/tests/decode.rs:374-397: region decode equals the
    # crop of the full decode.
    t = encode.config0(keep_pixels=True).tiles[0]
    full = np.frombuffer(oracle.decode(t.codestream, 1)[0], np.uint8).reshape(256, 256, 3)
    got, w, h = oracle.decode(t.codestream, 1, kind=1, roi=(13, 40, 101, 77))
    assert (w, h) == (101, 77)
    assert got == full[40:117, 13:114].tobytes()


def test_reduced_resolution_equals_forward_ll():
    # A Quarter decode of a gray tile equals the LL band two levels down of
    # the encoder's forward 5/3 plus the DC shift.
    rng = np.random.default_rng(5)
    px = rng.integers(0, 256, (64, 64), dtype=np.uint8)
    cs = encode.encode_lossless(px.reshape(-1), 64, 64, 1, 8, levels=3, cb_exp=3)
    got, w, h = oracle.decode(cs, 0, kind=2, denom=4)
    assert (w, h) == (16, 16)
    x = px.astype(np.int64) - 128

    def fwd(a):
        a = a.copy()
        n = a.shape[0]
        for i in range(1, n, 2):
            r = a[i + 1] if i + 1 < n else a[i - 1]
            a[i] -= (a[i - 1] + r) >> 1
        for i in range(0, n, 2):
            l = a[i - 1] if i - 1 >= 0 else a[i + 1]
            r = a[i + 1] if i + 1 < n else a[i - 1]
            a[i] += (l + r + 2) >> 2
        return a

    for _ in range(2):
        x = np.stack([fwd(x[:, c]) for c in range(x.shape[1])], axis=1)
        x = np.stack([fwd(x[r]) for r in range(x.shape[0])], axis=0)
        x = x[::2, ::2]
    want = np.clip(x + 128, 0, 255).astype(np.uint8)
    assert got == want.tobytes()
