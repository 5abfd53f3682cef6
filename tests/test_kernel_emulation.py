"""The decode kernels' CUDA source run on CPU threads (tests/kernel_emu):
every HT, classic (EBCOT), IDWT and pack kernel on the golden fixtures and
on seeded random reversible, irreversible and classic codestreams, built with AddressSanitizer, and
compared with the oracle (coefficients per code block, then pixels, exact).
Out-of-bounds accesses and parity breaks show up here without a GPU."""
import json
import pathlib
import shutil
import subprocess
import sys

import numpy as np
import pytest

from tests.helpers import (WIDE_BLOCKS, precinct_codestream, random_classic, random_codestream, random_irreversible,
                           wide_block_codestream)

EMU = pathlib.Path(__file__).parent / "kernel_emu"
ROOT = EMU.parents[1]
CSRC = ROOT / "signinum_b200" / "csrc"

pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")


@pytest.fixture(scope="module")
def emu(tmp_path_factory):
    out = tmp_path_factory.mktemp("kernel_emu")
    subprocess.run([sys.executable, str(EMU / "make_sources.py"), str(out)], check=True)
    flags = ["g++", "-std=c++20", "-O1", "-fsanitize=address", "-ffp-contract=off", f"-I{EMU}", f"-I{CSRC}",
             f"-I{ROOT / 'oracle'}"]
    units = [out / "ht_decode_emu.cpp", out / "idwt_pack_emu.cpp", out / "classic_emu.cpp", EMU / "emu_main.cpp",
             CSRC / "host" / "codestream.cpp",
             ROOT / "oracle" / "oracle.cpp", ROOT / "oracle" / "oracle_ht.cpp", ROOT / "oracle" / "oracle_ebcot.cpp",
             ROOT / "oracle" / "oracle_capi.cpp"]
    procs = [subprocess.Popen(flags + ["-c", str(u), "-o", str(out / (u.stem + ".o"))]) for u in units]
    assert all(p.wait() == 0 for p in procs)
    subprocess.run(flags + ["-o", str(out / "emu")] + [str(out / (u.stem + ".o")) for u in units] + ["-lpthread"],
                   check=True)
    return out


def run(emu, fmts, codestreams):
    paths = []
    for k, cs in enumerate(codestreams):
        p = emu / f"case_{fmts}_{k}.j2k"
        p.write_bytes(cs)
        paths.append(str(p))
    r = subprocess.run([str(emu / "emu"), fmts] + paths, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert r.stdout.strip().endswith("fails 0")


def test_golden_fixtures_through_emulated_kernels(emu):
    fx = json.loads((pathlib.Path(__file__).parent / "golden" / "openhtj2k.json").read_text())["fixtures"]
    run(emu, "03", [bytes.fromhex(f["j2k_hex"]) for f in fx.values()])


@pytest.mark.parametrize("kind", ["reversible", "irreversible", "classic"])
def test_random_codestreams_through_emulated_kernels(emu, kind):
    rng = np.random.default_rng({"reversible": 31, "irreversible": 97, "classic": 7}[kind])
    make = {"reversible": random_codestream, "irreversible": random_irreversible, "classic": random_classic}[kind]
    by_comps = {1: [], 3: []}
    while len(by_comps[1]) < 4 or len(by_comps[3]) < 4:
        cs, _, _, _, comps, _ = make(rng, max_side=100)
        by_comps[comps].append(cs)
    run(emu, "03", by_comps[1])  # Gray8, Gray16
    run(emu, "124", by_comps[3])  # Rgb8, Rgba8, Rgb16


def test_wide_code_blocks_through_emulated_kernels(emu):
    """HT blocks wider or higher than 64 (the VLC and MagSgn kernels' wide
    paths) under AddressSanitizer."""
    rng = np.random.default_rng(4200)
    by_comps = {1: [], 3: []}
    for cb in WIDE_BLOCKS:
        cs, _, _, _, comps, _ = wide_block_codestream(rng, cb, max_w=160, max_h=72)
        by_comps[comps].append(cs)
    if by_comps[1]:
        run(emu, "03", by_comps[1])
    if by_comps[3]:
        run(emu, "124", by_comps[3])


@pytest.mark.parametrize("kind", ["ht", "classic", "lossy"])
def test_precinct_partitions_through_emulated_kernels(emu, kind):
    """Precinct partitions through the product's host parser (which builds
    the job tables) and the emulated kernels."""
    rng = np.random.default_rng({"ht": 4400, "classic": 4401, "lossy": 4402}[kind])
    by_comps = {1: [], 3: []}
    while len(by_comps[1]) < 3 or len(by_comps[3]) < 3:
        cs, _, _, _, comps = precinct_codestream(rng, kind, max_side=90)
        by_comps[comps].append(cs)
    run(emu, "03", by_comps[1])
    run(emu, "124", by_comps[3])


def test_interior_strips_through_emulated_kernels(emu):
    """Levels wide enough for strips with no edge column (the 5/3 lifting's
    interior form: a strip from column 128 on that ends at least two columns
    before the level's edge), lossless RGB and gray, under AddressSanitizer."""
    from signinum_b200 import encode
    from tests.helpers import random_tile

    rng = np.random.default_rng(4500)
    by_comps = {1: [], 3: []}
    for w, h, comps, levels in [(300, 14, 3, 0), (390, 9, 3, 1), (517, 6, 1, 2), (640, 11, 3, 2), (259, 20, 1, 1)]:
        bd = 8 if comps == 3 else 12
        px = random_tile(rng, w, h, comps, bd, int(rng.integers(0, 2)))
        by_comps[comps].append(encode.encode_lossless(px.reshape(-1).view(np.uint8), w, h, comps, bd, levels=levels,
                                                      cb_exp=4, cb_exp_h=3))
    run(emu, "03", by_comps[1])
    run(emu, "124", by_comps[3])
