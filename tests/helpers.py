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
