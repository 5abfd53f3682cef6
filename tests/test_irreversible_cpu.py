"""The irreversible test inputs and the host parse of 9/7 codestreams (CPU)."""
import numpy as np

from oracle import oracle
from signinum_b200 import encode
from signinum_b200.j2k_cuda import inspect
from tests.helpers import random_irreversible


def test_irreversible_encode_round_trips_through_the_oracle():
    px = encode.he_rgb8(3, 96, 80)
    cs = encode.encode_irreversible(px, 96, 80, 3, 8, 1 / 512, levels=4)
    got, w, h = oracle.decode(cs, 1)
    assert (w, h) == (96, 80)
    err = np.abs(np.frombuffer(got, np.uint8).astype(int) - px.astype(int))
    assert err.mean() < 2.0 and err.max() < 24


def test_host_inspect_reports_irreversible():
    rng = np.random.default_rng(5)
    for _ in range(5):
        cs, _, w, h, comps, bd = random_irreversible(rng)
        info = inspect(cs)
        assert (info.dimensions, info.components, info.bit_depth) == ((w, h), comps, bd)
        assert info.reversible is False
