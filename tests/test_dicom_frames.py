"""DICOM encapsulated Pixel Data -> JPEG 2000 frames (sgn_dicom_frames),
the cases of the reference's own tests
(crates/signinum-j2k-metal/src/dicom.rs:462-599) plus malformed files; the
frames then decode bit-exactly (GPU)."""
import struct

import pytest

from oracle import oracle
from signinum_b200 import BackendRequest, Codec, Error, PixelFormat, dicom_frames, encode


def _item(payload: bytes) -> bytes:
    return b"\xfe\xff\x00\xe0" + struct.pack("<I", len(payload)) + payload


def _ov(tag: bytes, payload: bytes) -> bytes:
    # explicit VR OV element: tag, "OV", 2 reserved bytes, 32-bit length
    return tag + b"OV\x00\x00" + struct.pack("<I", len(payload)) + payload


def _dicom(bot: bytes, fragments, ext_offsets=None, ext_lengths=None, header=b"DICM" * 8) -> bytes:
    b = bytearray(header)
    if ext_offsets is not None:
        b += _ov(b"\xe0\x7f\x01\x00", b"".join(struct.pack("<Q", o) for o in ext_offsets))
    if ext_lengths is not None:
        b += _ov(b"\xe0\x7f\x02\x00", b"".join(struct.pack("<Q", n) for n in ext_lengths))
    b += b"\xe0\x7f\x10\x00" + b"OB\x00\x00" + b"\xff\xff\xff\xff"  # Pixel Data, undefined length
    b += _item(bot)
    for f in fragments:
        b += _item(f)
    b += b"\xfe\xff\xdd\xe0" + b"\x00\x00\x00\x00"
    return bytes(b)


def test_empty_basic_offset_table_gives_one_frame_per_fragment():
    assert dicom_frames(_dicom(b"", [b"abcd", b"ef"])) == [b"abcd", b"ef"]


def test_basic_offset_table_groups_fragments():
    # Item offsets from the first fragment's item tag: 0, 12, 22.
    bot = struct.pack("<II", 0, 18)
    assert dicom_frames(_dicom(bot, [b"abcd", b"ef", b"gh"])) == [b"abcdef", b"gh"]


def test_extended_offset_table_lengths_trim_padding():
    frames = dicom_frames(_dicom(b"", [b"abcd", b"efgh"], ext_offsets=[0, 12], ext_lengths=[3, 2]))
    assert frames == [b"abc", b"ef"]


def test_limit_stops_early():
    assert dicom_frames(_dicom(b"", [b"a1", b"b2", b"c3"]), limit=2) == [b"a1", b"b2"]
    bot = struct.pack("<III", 0, 10, 20)
    assert dicom_frames(_dicom(bot, [b"a1", b"b2", b"c3"]), limit=1) == [b"a1"]
    assert dicom_frames(_dicom(b"", [b"a1"]), limit=0) == []


@pytest.mark.parametrize("blob,status", [
    (b"no pixel data here" * 4, 4),                                                # Pixel Data not found
    (b"DICM" + b"\xe0\x7f\x10\x00OB\x00\x00" + struct.pack("<I", 16) + b"\x00" * 16, 1),  # not encapsulated
    (_dicom(b"", [b"abcd"])[:-12], 3),                                             # truncated item
    (_dicom(struct.pack("<II", 12, 0), [b"abcd", b"ef"]), 4),                      # offsets not increasing
    (_dicom(b"\x00\x00", [b"abcd"]), 4),                                           # BOT not a multiple of 4
])
def test_malformed_files(blob, status):
    with pytest.raises(Error) as e:
        dicom_frames(blob)
    assert e.value.status == status


@pytest.mark.gpu
def test_dicom_frames_decode_bit_exact():
    tiles = encode.config2(n=4).tiles
    # Split every codestream into two fragments; group them with a Basic Offset Table.
    frags, bot, at = [], [], 0
    for t in tiles:
        cs = t.codestream
        h = len(cs) // 2
        bot.append(at)
        for part in (cs[:h], cs[h:]):
            frags.append(part)
            at += 8 + len(part)
    frames = dicom_frames(_dicom(b"".join(struct.pack("<I", o) for o in bot), frags))
    assert frames == [t.codestream for t in tiles]
    surfaces = Codec.decode_tiles_to_device(frames, PixelFormat.Rgb8, BackendRequest.Cuda)
    for t, s in zip(tiles, surfaces):
        assert s.to_bytes() == oracle.decode(t.codestream, int(PixelFormat.Rgb8))[0]
