"""Shared helpers for the parity tests."""
import numpy as np

from signinum_b200 import encode


def random_tile(rng, w, h, comps, bd, kind):
    if bd <= 8:
        if kind == 0:
            px = rng.integers(0, 1 << bd, (h, w, comps), dtype=np.uint8)
        elif kind == 1:
            px = np.clip(np.round(rng.normal(1 << (bd - 1), 5, (h, w, comps))), 0, (1 << bd) - 1).astype(np.uint8)
        else:
            px = np.full((h, w, comps), rng.integers(0, 1 << bd), np.uint8)
    else:
        if kind == 2:
            px = np.full((h, w, comps), rng.integers(0, 1 << bd), "<u2")
        else:
            px = rng.integers(0, 1 << bd, (h, w, comps)).astype("<u2")
    return np.ascontiguousarray(px)


def random_codestream(rng, max_side=80):
    w = int(rng.integers(1, max_side))
    h = int(rng.integers(1, max_side))
    comps = int(rng.choice([1, 3]))
    bd = int(rng.choice([8, 8, 12, 16])) if comps == 1 else int(rng.choice([8, 8, 8, 10]))
    kind = int(rng.integers(0, 3))
    px = random_tile(rng, w, h, comps, bd, kind)
    cbw = int(rng.integers(0, 5))
    cbh = int(rng.integers(0, 5))
    if cbw + cbh > 8:
        cbh = 8 - cbw
    cs = encode.encode_lossless(px.reshape(-1).view(np.uint8), w, h, comps, bd, levels=int(rng.integers(0, 7)),
                                cb_exp=cbw, cb_exp_h=cbh, progression=int(rng.choice([0, 1, 2, 3, 4])),
                                sop_eph=bool(rng.integers(0, 2)))
    return cs, px, w, h, comps, bd


# Code-block shapes beyond 64 on a side (exponents over the 4-sample base),
# within JPEG 2000's limits (at most 1024 on a side, w h <= 4096).
WIDE_BLOCKS = [(5, 3), (6, 2), (7, 1), (8, 0), (3, 5), (0, 8), (5, 1)]


def wide_block_codestream(rng, cb, max_w=300, max_h=140):
    """A seeded lossless HT codestream whose code blocks have the exponents
    cb = (width, height): 128x32 .. 1024x4 and 4x1024 blocks."""
    w = int(rng.integers(40, max_w))
    h = int(rng.integers(12, max_h))
    comps = int(rng.choice([1, 3]))
    bd = int(rng.choice([8, 12, 16])) if comps == 1 else 8
    px = random_tile(rng, w, h, comps, bd, int(rng.integers(0, 2)))
    cs = encode.encode_lossless(px.reshape(-1).view(np.uint8), w, h, comps, bd, levels=int(rng.integers(0, 4)),
                                cb_exp=cb[0], cb_exp_h=cb[1], progression=int(rng.choice([0, 2, 4])))
    return cs, px, w, h, comps, bd


def precinct_codestream(rng, kind, max_side=200):
    """A seeded codestream cut into precincts of 2^PPx x 2^PPy (2 .. 256) in
    any progression, its packets split over 1-6 tile-parts: kind "ht"
    (lossless, with or without TLM), "classic" (lossless, 1-3 layers, random
    code-block styles) or "lossy" (9/7).  Returns the codestream, the pixels,
    width, height and components."""
    w = int(rng.integers(1, max_side))
    h = int(rng.integers(1, max_side))
    comps = int(rng.choice([1, 3]))
    px = random_tile(rng, w, h, comps, 8, int(rng.integers(0, 2)))
    pp = (int(rng.integers(1, 9)), int(rng.integers(1, 9)))
    cbw = int(rng.integers(0, 5))
    cbh = min(int(rng.integers(0, 5)), 8 - cbw)
    kw = dict(levels=int(rng.integers(0, 6)), cb_exp=cbw, cb_exp_h=cbh, progression=int(rng.integers(0, 5)),
              precincts=pp, tile_parts=int(rng.integers(1, 7)))
    flat = px.reshape(-1)
    if kind == "ht":
        cs = encode.encode_lossless(flat, w, h, comps, 8, write_tlm=bool(rng.integers(0, 2)), **kw)
    elif kind == "classic":
        cs = encode.encode_classic(flat, w, h, comps, 8, style=int(rng.choice([0, 0x01, 0x04, 0x05, 0x2F])),
                                   layers=int(rng.integers(1, 4)), **kw)
    else:
        cs = encode.encode_irreversible(flat, w, h, comps, 8, **kw)
    return cs, px, w, h, comps


def _box(btype: bytes, payload: bytes, form: str = "short") -> bytes:
    """One JP2 box: 'short' (32-bit length), 'long' (extended 64-bit length)
    or 'to_end' (length 0: the box runs to the end of the file)."""
    import struct

    if form == "long":
        return struct.pack(">I", 1) + btype + struct.pack(">Q", 16 + len(payload)) + payload
    if form == "to_end":
        return struct.pack(">I", 0) + btype + payload
    return struct.pack(">I", 8 + len(payload)) + btype + payload


def jp2_wrap(codestream: bytes, width: int, height: int, comps: int, bit_depth: int = 8, colr_enum=None,
             icc: bool = False, extra_jp2h: bytes = b"", jp2c_form: str = "short", with_ihdr: bool = True,
             order=("jP", "ftyp", "jp2h", "jp2c")) -> bytes:
    """A JP2 file around a raw codestream (ISO/IEC 15444-1 Annex I boxes)."""
    import struct

    if colr_enum is None:
        colr_enum = 16 if comps == 3 else 17
    ihdr = _box(b"ihdr", struct.pack(">IIHBBBB", height, width, comps, bit_depth - 1, 7, 0, 0))
    colr = _box(b"colr", bytes([2, 0, 0]) + b"\x00" * 8) if icc else \
        _box(b"colr", bytes([1, 0, 0]) + struct.pack(">I", colr_enum))
    parts = {
        "jP": _box(b"jP  ", b"\x0d\x0a\x87\x0a"),
        "ftyp": _box(b"ftyp", b"jp2 " + struct.pack(">I", 0) + b"jp2 "),
        "jp2h": _box(b"jp2h", (ihdr if with_ihdr else b"") + colr + extra_jp2h),
        "jp2c": _box(b"jp2c", codestream, jp2c_form),
    }
    return b"".join(parts[k] for k in order)


def random_irreversible(rng, max_side=80):
    """A seeded lossy 9/7 codestream (ICT for RGB, expounded quantisation)."""
    w = int(rng.integers(1, max_side))
    h = int(rng.integers(1, max_side))
    comps = int(rng.choice([1, 3]))
    bd = int(rng.choice([8, 8, 12, 16])) if comps == 1 else int(rng.choice([8, 8, 8, 10]))
    px = random_tile(rng, w, h, comps, bd, int(rng.integers(0, 3)))
    cbw = int(rng.integers(0, 5))
    cbh = min(int(rng.integers(0, 5)), 8 - cbw)
    step = float(rng.choice([1 / 16, 1 / 100, 1 / 256, 1 / 1000, 3 / 4096]))
    cs = encode.encode_irreversible(px.reshape(-1).view(np.uint8), w, h, comps, bd, step,
                                    levels=int(rng.integers(0, 7)), cb_exp=cbw, cb_exp_h=cbh,
                                    use_mct=bool(rng.integers(0, 4)), progression=int(rng.choice([0, 1, 2, 3, 4])))
    return cs, px, w, h, comps, bd


CLASSIC_STYLES = [0, 0x01, 0x02, 0x04, 0x08, 0x20, 0x05, 0x0D, 0x2F]


def random_classic(rng, max_side=80):
    """A seeded classic (EBCOT) codestream: random code-block style, lossless
    5/3 or lossy 9/7."""
    w = int(rng.integers(1, max_side))
    h = int(rng.integers(1, max_side))
    comps = int(rng.choice([1, 3]))
    bd = int(rng.choice([8, 8, 12, 16])) if comps == 1 else int(rng.choice([8, 8, 8, 10]))
    px = random_tile(rng, w, h, comps, bd, int(rng.integers(0, 3)))
    cbw = int(rng.integers(0, 9))  # classic blocks up to 1024 wide (w h <= 4096)
    cbh = min(int(rng.integers(0, 9)), 8 - cbw)
    irr = bool(rng.integers(0, 2))
    cs = encode.encode_classic(px.reshape(-1).view(np.uint8), w, h, comps, bd,
                               style=int(rng.choice(CLASSIC_STYLES)), irreversible=irr,
                               relative_step=float(rng.choice([1 / 64, 1 / 256, 1 / 1000])),
                               levels=int(rng.integers(0, 7)), cb_exp=cbw, cb_exp_h=cbh,
                               use_mct=bool(rng.integers(0, 4)), progression=int(rng.choice([0, 1, 2, 3, 4])),
                               layers=int(rng.choice([1, 1, 2, 3, 5])))
    return cs, px, w, h, comps, bd
