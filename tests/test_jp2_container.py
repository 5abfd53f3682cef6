"""JP2 input (crates/signinum-j2k/src/parse/boxes.rs): the container is
parsed on the host, its codestream decoded like a raw one; malformed files
and colour specifications the path cannot map report the reference's error
kinds.  CPU part: the oracle and the host parser; GPU part: the decode."""
import ctypes

import numpy as np
import pytest

from oracle import oracle
from signinum_b200 import BackendRequest, Error, J2kDecoder, PixelFormat, encode, inspect
from tests.helpers import _box, jp2_wrap


@pytest.fixture(scope="module")
def tile():
    return encode.config0().tiles[0]


def _files(t):
    cs = t.codestream
    good = {
        "plain": jp2_wrap(cs, t.width, t.height, 3),
        "jp2c_to_end": jp2_wrap(cs, t.width, t.height, 3, jp2c_form="to_end"),
        "jp2c_extended_length": jp2_wrap(cs, t.width, t.height, 3, jp2c_form="long"),
        "unknown_boxes_skipped": jp2_wrap(cs, t.width, t.height, 3, extra_jp2h=_box(b"res ", b"\x00" * 10)),
    }
    bad = {
        # (file, status): 1 unsupported, 3 truncated, 4 decode
        "missing_ihdr": (jp2_wrap(cs, t.width, t.height, 3, with_ihdr=False), 4),
        "jp2c_before_jp2h": (jp2_wrap(cs, t.width, t.height, 3, order=("jP", "ftyp", "jp2c", "jp2h")), 4),
        "ftyp_missing": (jp2_wrap(cs, t.width, t.height, 3, order=("jP", "jp2h", "jp2c")), 4),
        "truncated_box": (jp2_wrap(cs, t.width, t.height, 3)[:-100], 3),
        "not_j2k_at_all": (b"GIF89a" + b"\x00" * 64, 1),
        "icc_profile": (jp2_wrap(cs, t.width, t.height, 3, icc=True), 1),
        "sycc": (jp2_wrap(cs, t.width, t.height, 3, colr_enum=18), 1),
        "greyscale_colr_on_rgb": (jp2_wrap(cs, t.width, t.height, 3, colr_enum=17), 1),
        "palette_box": (jp2_wrap(cs, t.width, t.height, 3, extra_jp2h=_box(b"pclr", b"\x00" * 8)), 1),
    }
    return good, bad


def test_oracle_decodes_jp2_like_the_raw_codestream(tile):
    want = oracle.decode(tile.codestream, int(PixelFormat.Rgb8))
    good, bad = _files(tile)
    for name, f in good.items():
        assert oracle.decode(f, int(PixelFormat.Rgb8)) == want, name
    for name, (f, status) in bad.items():
        with pytest.raises(oracle.OracleError) as e:
            oracle.decode(f, int(PixelFormat.Rgb8))
        assert e.value.status == status, name


def test_host_inspect_reads_jp2(tile):
    raw = inspect(tile.codestream)
    good, bad = _files(tile)
    for name, f in good.items():
        assert inspect(f).dimensions == raw.dimensions, name
    for name in ("missing_ihdr", "jp2c_before_jp2h", "truncated_box", "not_j2k_at_all"):
        f, status = bad[name]
        with pytest.raises(Error) as e:
            inspect(f)
        assert e.value.status == status, name


@pytest.mark.gpu
def test_gpu_decodes_jp2_and_reports_oracle_errors(tile):
    want = oracle.decode(tile.codestream, int(PixelFormat.Rgb8))[0]
    good, bad = _files(tile)
    for name, f in good.items():
        s = J2kDecoder(f).decode_to_device(PixelFormat.Rgb8, BackendRequest.Cuda)
        assert s.to_bytes() == want, name
    for name, (f, status) in bad.items():
        with pytest.raises(Error) as e:
            J2kDecoder(f).decode_to_device(PixelFormat.Rgb8, BackendRequest.Cuda)
        assert e.value.status == status, name
