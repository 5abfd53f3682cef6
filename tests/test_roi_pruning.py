"""Region requests decode only the code blocks their region needs
(RoiPlan::build / code_block_required, crates/signinum-j2k-native/src/j2c/roi.rs:18-270),
checked on the host through sgn_j2k_request_blocks (no GPU): a small region of
a large tile decodes a small fraction of its blocks; full, reduced and edge
regions decode them all, as the reference plans them."""
import ctypes

import numpy as np
import pytest

from signinum_b200 import _native, encode
from signinum_b200._native import SgnRequest


def _blocks(cs, fmt, kind=0, rect=(0, 0, 0, 0), d=1):
    arr = np.frombuffer(cs, np.uint8)
    req = SgnRequest(kind, *rect, d)
    dec, tot = ctypes.c_uint64(), ctypes.c_uint64()
    st = _native.cuda_lib().sgn_j2k_request_blocks(arr.ctypes.data, arr.nbytes, fmt, ctypes.byref(req),
                                                    ctypes.byref(dec), ctypes.byref(tot))
    assert st == 0, _native.last_error()
    return dec.value, tot.value


@pytest.fixture(scope="module")
def big_tile():
    px = encode.he_rgb8(91, 1024, 1024, 12.0)
    return encode.encode_lossless(px, 1024, 1024, 3, 8, levels=6, cb_exp=4)


def test_small_region_of_a_large_tile_decodes_few_blocks(big_tile):
    full, total = _blocks(big_tile, 1)
    assert full == total > 700
    d, t = _blocks(big_tile, 1, 1, (400, 300, 64, 64))
    assert t == total
    # 64x64 of 1024x1024: the blocks under the window plus the 16-sample
    # margin of every level, about 3 blocks a side per band at the finest level.
    assert d < total // 8, (d, total)
    d2, _ = _blocks(big_tile, 1, 1, (400, 300, 256, 256))
    assert d < d2 < total // 2


def test_region_scaled_prunes_at_the_reduced_resolution(big_tile):
    # A quarter-resolution decode keeps 4 of 6 levels; a 64x64 region of the
    # 256x256 image still prunes.
    d_all, t = _blocks(big_tile, 1, 2, (0, 0, 0, 0), 4)
    assert d_all == t
    # Half resolution keeps 5 levels (210 blocks): a small region needs few.
    d, _ = _blocks(big_tile, 1, 3, (40, 40, 32, 32), 4)
    assert d < t, (d, t)
    d2, t2 = _blocks(big_tile, 1, 3, (0, 0, 8, 8), 2)
    assert t2 > t and d2 < t2 // 3, (d2, t2)


@pytest.mark.parametrize("rect", [(0, 0, 1024, 1024), (960, 10, 64, 64), (10, 960, 64, 64), (0, 0, 1024, 1)])
def test_regions_reaching_the_right_or_bottom_edge_decode_everything(big_tile, rect):
    d, t = _blocks(big_tile, 1, 1, rect)
    assert d == t


def test_region_at_the_origin_prunes(big_tile):
    d, t = _blocks(big_tile, 1, 1, (0, 0, 8, 8))
    assert 0 < d < t // 8, (d, t)


def test_invalid_region_is_reported():
    px = encode.he_rgb8(3, 128, 128, 6.0)
    cs = encode.encode_lossless(px, 128, 128, 3, 8, levels=3, cb_exp=3)
    arr = np.frombuffer(cs, np.uint8)
    req = SgnRequest(1, 100, 100, 64, 64, 1)
    dec, tot = ctypes.c_uint64(), ctypes.c_uint64()
    st = _native.cuda_lib().sgn_j2k_request_blocks(arr.ctypes.data, arr.nbytes, 1, ctypes.byref(req),
                                                    ctypes.byref(dec), ctypes.byref(tot))
    assert st == 5  # SGN_ERR_REGION
