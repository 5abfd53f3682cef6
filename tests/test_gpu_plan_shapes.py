"""GPU: every launch shape of a batch plan (grid or persistent work-queue
kernels), graph replay and the autotuner's choice decode bit-exactly."""
import pytest

from oracle import oracle
from signinum_b200 import PixelFormat, encode
from signinum_b200.plan import Plan

pytestmark = pytest.mark.gpu

SHAPES = [
    (128, 8, 0, 0),  # default: one block / unit per warp
    (64, 4, 0, 0),
    (128, 8, 1, 3),  # persistent MagSgn (1 block per grab), IDWT and pack queues
    (96, 4, 4, 1),   # persistent MagSgn, 4 blocks per grab, IDWT queue
    (32, 1, 2, 2),   # pack queue
]


@pytest.fixture(scope="module")
def batch():
    # Uneven tiles (sizes, block sizes, near-blank) to exercise the queues.
    return encode.config2(n=10).tiles


def _want(tiles):
    return [oracle.decode(t.codestream, int(PixelFormat.Rgb8))[0] for t in tiles]


@pytest.mark.parametrize("shape", SHAPES, ids=[f"vlc{a}_ms{b}x{c}_dwtq{d}" for a, b, c, d in SHAPES])
def test_launch_shapes_are_bit_exact(batch, shape):
    want = _want(batch)
    plan = Plan([t.codestream for t in batch], int(PixelFormat.Rgb8))
    plan.set_launch_shape(*shape)
    for rep in range(3):  # eager, graph capture, graph replay
        plan.execute_async()
        st, per = plan.wait()
        assert st == 0 and per == [0] * len(batch)
        for i in (0, len(batch) // 2, len(batch) - 1):
            assert plan.download(i) == want[i], f"tile {i}, execution {rep}"
    assert [plan.download(i) for i in range(len(batch))] == want
    plan.destroy()


def test_autotune_keeps_output_and_is_reused(batch):
    want = _want(batch)
    plan = Plan([t.codestream for t in batch], int(PixelFormat.Rgb8))
    rep = plan.autotune(2)
    assert rep["vlc_threads"] in (64, 128) and rep["ms_warps"] in (4, 8) and rep["dwt_queue"] in (0, 1, 2, 3)
    assert rep["vlc_ms"] > 0 and rep["ms_ms"] > 0 and rep["dwt_ms"] > 0
    assert [plan.download(i) for i in range(len(batch))] == want
    for _ in range(3):
        plan.execute_async()
    st, _ = plan.wait()
    assert st == 0 and [plan.download(i) for i in range(len(batch))] == want
    plan.destroy()


@pytest.mark.parametrize("shift", [(-4, -4), (-3, -2), (-2, -2), (-1, -1), (1, 1), (-1, 1), (1, 0)])
def test_dwt_tile_shapes_are_bit_exact(shift):
    """Rows per IDWT / pack unit quartered, halved or doubled, on reversible and
    irreversible tiles and on pruned region decodes (windowed levels)."""
    from signinum_b200.j2k_cuda import Rect, _request

    tiles = encode.config2(n=6).tiles
    lossy = encode.encode_irreversible(encode.he_rgb8(5, 300, 200, 9.0), 300, 200, 3, 8, 1 / 256, levels=4, cb_exp=4)
    big = tiles[[t.width for t in tiles].index(max(t.width for t in tiles))]
    roi = Rect(big.width // 3, big.height // 4, 77, 45)
    inputs = [t.codestream for t in tiles] + [lossy, big.codestream]
    reqs = [_request(0)] * (len(inputs) - 1) + [_request(1, roi)]
    want = [oracle.decode(c, int(PixelFormat.Rgb8))[0] for c in inputs[:-1]]
    want.append(oracle.decode(big.codestream, int(PixelFormat.Rgb8), 1, (roi.x, roi.y, roi.w, roi.h), 1)[0])
    plan = Plan(inputs, int(PixelFormat.Rgb8), requests=reqs)
    plan.set_tile_shape(*shift)
    for _ in range(3):
        plan.execute_async()
        st, _ = plan.wait()
        assert st == 0
        assert [plan.download(i) for i in range(len(inputs))] == want
    plan.destroy()


def test_autotuned_tile_shape_applies_to_the_next_plan_of_the_same_shape(batch):
    want = _want(batch)
    a = Plan([t.codestream for t in batch], int(PixelFormat.Rgb8))
    rep = a.autotune(2)
    assert rep["idwt_seg_shift"] in range(-4, 2) and rep["pack_seg_shift"] in range(-4, 2)
    assert rep["vlc_lanes"] in (1, 2, 4, 8, 16, 32) and rep["vlc_outline"] in (0, 1)
    assert rep["ht_fused"] in (0, 1) and rep["idwt_lean"] in (0, 1)
    a.destroy()
    b = Plan([t.codestream for t in batch], int(PixelFormat.Rgb8))
    b.execute_async()
    st, _ = b.wait()
    assert st == 0 and [b.download(i) for i in range(len(batch))] == want
    b.destroy()


@pytest.mark.parametrize("form", [0, 1, 2])
def test_cleanup_forms_are_bit_exact(form):
    """The HT cleanup as two kernels over all blocks (0), as one kernel whose
    MagSgn warp follows each block's VLC chain row by row (1), or chosen by
    block count (2): refinement passes, blocks wider than 64 and narrow ones,
    in eager runs and graph replays."""
    import json
    import pathlib

    import numpy as np

    from tests.helpers import random_codestream, wide_block_codestream

    rng = np.random.default_rng(5300)
    rgb, gray = [encode.config0().tiles[0].codestream], []
    fx = json.loads((pathlib.Path(__file__).parent / "golden" / "openhtj2k.json").read_text())["fixtures"]
    gray.append(bytes.fromhex(fx["openhtj2k_ds0_ht_12_b11"]["j2k_hex"]))
    while len(rgb) < 5 or len(gray) < 4:
        cs, _, _, _, comps, _ = random_codestream(rng)
        (rgb if comps == 3 else gray).append(cs)
    for cb in [(5, 3), (0, 8)]:  # 128x32 and 4x1024 blocks
        cs, _, _, _, comps, _ = wide_block_codestream(rng, cb, max_w=200, max_h=90)
        (rgb if comps == 3 else gray).append(cs)
    for inputs, fmt in [(rgb, PixelFormat.Rgb8), (gray, PixelFormat.Gray8)]:
        want = [oracle.decode(c, int(fmt))[0] for c in inputs]
        plan = Plan(inputs, int(fmt))
        plan.set_cleanup_form(form)
        for rep in range(3):
            plan.execute_async()
            st, per = plan.wait()
            assert st == 0 and per == [0] * len(inputs)
            assert [plan.download(i) for i in range(len(inputs))] == want, f"form {form}, execution {rep}"
        plan.destroy()
