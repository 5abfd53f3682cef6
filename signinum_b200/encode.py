"""Lossless HTJ2K encode and the seeded synthetic workloads.

encode_lossless() stands where the reference's lossless facade stands
(encode_j2k_lossless with HighThroughput block coding,
crates/signinum-j2k/src/encode.rs:166-188).  The workload builders produce
the tiles the benchmark and parity tests decode; every tile is a pure
function of (master seed, workload, tile index).
"""
from __future__ import annotations

import ctypes
import os
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field
from typing import List

import numpy as np

from . import _native
from ._native import SgnEncodeOptions

MASTER_SEED = 0x51674E01


def _mix(*parts) -> int:
    """splitmix64 over the parts: per-tile seeds from (master, workload, index)."""
    x = 0
    for p in parts:
        x = (x + (p & 0xFFFFFFFFFFFFFFFF) + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        z = x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        x = z ^ (z >> 31)
    return x


def _encode(call, cap: int) -> bytes:
    """Runs an encoder entry point into a buffer of `cap` bytes; when that is
    too small (-4, the needed length reported) once more with that length."""
    for _ in range(2):
        out = np.zeros(cap, np.uint8)
        n = ctypes.c_size_t()
        rc = call(out.ctypes.data, cap, ctypes.byref(n))
        if rc == -4 and n.value > cap:
            cap = n.value
            continue
        if rc != 0:
            raise ValueError(f"encode failed ({rc})")
        return out[: n.value].tobytes()
    raise ValueError("encode failed (-4)")


def encode_lossless(pixels: np.ndarray, width: int, height: int, components: int, bit_depth: int,
                    levels: int = 5, cb_exp: int = 4, use_mct: bool = True, progression: int = 0,
                    sop_eph: bool = False, write_tlm: bool = False, cb_exp_h: int | None = None,
                    precincts: tuple = (0, 0), tile_parts: int = 1) -> bytes:
    """Encodes interleaved samples (u8, or little-endian u16 for depths > 8).
    precincts: (PPx, PPy) exponents of every resolution, (0, 0) for one
    precinct per resolution; tile_parts: tile-parts the packets are split
    into."""
    px = np.ascontiguousarray(pixels)
    opts = SgnEncodeOptions(levels, cb_exp, cb_exp if cb_exp_h is None else cb_exp_h, int(use_mct), progression,
                            int(write_tlm), int(sop_eph), precincts[0], precincts[1], tile_parts)
    return _encode(lambda out, cap, n: _native.encode_lib().sgn_j2k_encode_lossless(
        px.ctypes.data, width, height, components, bit_depth, ctypes.byref(opts), out, cap, n), px.nbytes * 2 + 65536)


def encode_irreversible(pixels: np.ndarray, width: int, height: int, components: int, bit_depth: int,
                        relative_step: float = 1.0 / 256, levels: int = 5, cb_exp: int = 4, use_mct: bool = True,
                        progression: int = 0, cb_exp_h: int | None = None, precincts: tuple = (0, 0),
                        tile_parts: int = 1) -> bytes:
    """Lossy 9/7 codestream (ICT, scalar expounded quantisation) for the
    irreversible decode path's tests; same sample layout as encode_lossless."""
    px = np.ascontiguousarray(pixels)
    opts = SgnEncodeOptions(levels, cb_exp, cb_exp if cb_exp_h is None else cb_exp_h, int(use_mct), progression, 0, 0,
                            precincts[0], precincts[1], tile_parts)
    return _encode(lambda out, cap, n: _native.encode_lib().sgn_j2k_encode_irreversible(
        px.ctypes.data, width, height, components, bit_depth, ctypes.byref(opts), relative_step, out, cap, n),
        px.nbytes * 2 + 65536)


def encode_classic(pixels: np.ndarray, width: int, height: int, components: int, bit_depth: int, style: int = 0,
                   irreversible: bool = False, relative_step: float = 1.0 / 256, levels: int = 5, cb_exp: int = 4,
                   use_mct: bool = True, progression: int = 0, cb_exp_h: int | None = None, layers: int = 1,
                   precincts: tuple = (0, 0), tile_parts: int = 1) -> bytes:
    """Classic (EBCOT Tier-1) codestream with code-block style bits `style`,
    lossless 5/3 or (irreversible) lossy 9/7, `layers` quality layers; same
    sample layout as encode_lossless."""
    px = np.ascontiguousarray(pixels)
    opts = SgnEncodeOptions(levels, cb_exp, cb_exp if cb_exp_h is None else cb_exp_h, int(use_mct), progression, 0, 0,
                            precincts[0], precincts[1], tile_parts)
    return _encode(lambda out, cap, n: _native.encode_lib().sgn_j2k_encode_classic(
        px.ctypes.data, width, height, components, bit_depth, ctypes.byref(opts), style, int(irreversible),
        relative_step, layers, out, cap, n), px.nbytes * 3 + 65536)


def he_rgb8(seed: int, width: int, height: int, sigma: float = 6.0) -> np.ndarray:
    out = np.zeros(width * height * 3, np.uint8)
    _native.encode_lib().sgn_synth_he_rgb8(seed, width, height, sigma, out.ctypes.data)
    return out


def blank_rgb8(seed: int, width: int, height: int) -> np.ndarray:
    out = np.zeros(width * height * 3, np.uint8)
    _native.encode_lib().sgn_synth_blank_rgb8(seed, width, height, out.ctypes.data)
    return out


def fluor_gray16(seed: int, width: int, height: int) -> np.ndarray:
    out = np.zeros(width * height * 2, np.uint8)
    _native.encode_lib().sgn_synth_fluor_gray16(seed, width, height, out.ctypes.data)
    return out


@dataclass
class Tile:
    codestream: bytes
    width: int
    height: int
    components: int
    bit_depth: int
    levels: int
    cb: int
    kind: str
    pixels: np.ndarray | None = None


@dataclass
class Workload:
    name: str
    tiles: List[Tile] = field(default_factory=list)

    def pixels(self) -> int:
        return sum(t.width * t.height for t in self.tiles)

    def coded_bytes(self) -> int:
        return sum(len(t.codestream) for t in self.tiles)


def _pool():
    return ThreadPoolExecutor(max_workers=max(1, min(32, os.cpu_count() or 1)))


def _he_tile(widx: int, i: int, side: int, sigma: float, levels: int, cb_exp: int, keep: bool, blank=False,
             lossy_step: float | None = None, classic_style: int | None = None) -> Tile:
    seed = _mix(MASTER_SEED, widx, i)
    px = blank_rgb8(seed, side, side) if blank else he_rgb8(seed, side, side, sigma)
    if classic_style is not None:
        cs = encode_classic(px, side, side, 3, 8, style=classic_style, levels=levels, cb_exp=cb_exp)
    elif lossy_step is None:
        cs = encode_lossless(px, side, side, 3, 8, levels=levels, cb_exp=cb_exp)
    else:
        cs = encode_irreversible(px, side, side, 3, 8, lossy_step, levels=levels, cb_exp=cb_exp)
    return Tile(cs, side, side, 3, 8, levels, 1 << (cb_exp + 2), "blank" if blank else "he", px if keep else None)


def config0(keep_pixels=False) -> Workload:
    """One 256x256 RGB8 H&E-like tile, 5 levels, 64x64 code blocks, RCT."""
    return Workload("c0_rgb8_256x256", [_he_tile(0, 0, 256, 6.0, 5, 4, keep_pixels)])


def config1(n=256, side=512, keep_pixels=False) -> Workload:
    """256 tiles of 512x512 RGB8 (H&E-like, sigma 6), 5 levels, 64x64 blocks."""
    with _pool() as ex:
        tiles = list(ex.map(lambda i: _he_tile(1, i, side, 6.0, 5, 4, keep_pixels), range(n)))
    return Workload(f"c1_rgb8_{n}x{side}x{side}", tiles)


def config1_irreversible(n=256, side=512, step=1 / 256, keep_pixels=False) -> Workload:
    """The uniform batch of config1 coded lossy: ICT, 9/7, 5 levels, 64x64
    blocks, every band quantised with relative step `step`."""
    with _pool() as ex:
        tiles = list(ex.map(lambda i: _he_tile(5, i, side, 6.0, 5, 4, keep_pixels, lossy_step=step), range(n)))
    return Workload(f"c1i_rgb8_{n}x{side}x{side}_97", tiles)


def config1_classic(n=256, side=512, style=0, keep_pixels=False) -> Workload:
    """The uniform batch of config1 coded with classic (EBCOT) Tier-1 code
    blocks (code-block style bits `style`), lossless 5/3, RCT."""
    with _pool() as ex:
        tiles = list(ex.map(lambda i: _he_tile(6, i, side, 6.0, 5, 4, keep_pixels, classic_style=style), range(n)))
    return Workload(f"c1c_rgb8_{n}x{side}x{side}_ebcot", tiles)


def config2(n=1024, keep_pixels=False, indices=None) -> Workload:
    """1024 uneven RGB8 tiles: sides {128,256,512,1024}, noise sigma U[0,30],
    20% near-blank, levels 3..6 by side, 32x32 or 64x64 blocks.  With
    `indices`, only those tiles of the n-tile list (each tile is a pure
    function of n and its index)."""
    rng = np.random.default_rng(_mix(MASTER_SEED, 2) & 0xFFFFFFFF)
    sides = rng.choice([128, 256, 512, 1024], size=n)
    sigmas = rng.uniform(0, 30, size=n)
    blank = rng.uniform(0, 1, size=n) < 0.2
    cbs = rng.choice([3, 4], size=n)
    lv = {128: 3, 256: 4, 512: 5, 1024: 6}

    def one(i):
        s = int(sides[i])
        return _he_tile(2, i, s, float(sigmas[i]), lv[s], int(cbs[i]), keep_pixels, bool(blank[i]))

    with _pool() as ex:
        tiles = list(ex.map(one, range(n) if indices is None else indices))
    return Workload(f"c2_rgb8_uneven_{n}", tiles)


def config3(n=128, side=2048, keep_pixels=False) -> Workload:
    """128 single-component u16 2048x2048 fluorescence-like tiles, 6 levels, 64x64 blocks."""

    def one(i):
        seed = _mix(MASTER_SEED, 3, i)
        px = fluor_gray16(seed, side, side)
        cs = encode_lossless(px, side, side, 1, 16, levels=6, cb_exp=4, use_mct=False)
        return Tile(cs, side, side, 1, 16, 6, 64, "fluor", px if keep_pixels else None)

    with _pool() as ex:
        tiles = list(ex.map(one, range(n)))
    return Workload(f"c3_gray16_{n}x{side}x{side}", tiles)


def config4_pool(n=4096) -> Workload:
    """The serving pool: 4096 tiles drawn as in config2."""
    w = config2(n)
    w.name = f"c4_pool_{n}"
    return w
