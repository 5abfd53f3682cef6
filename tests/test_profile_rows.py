"""Environment-gated profiling rows in the reference's format
(crates/signinum-profile/src/lib.rs: SIGNINUM_GPU_ROUTE_PROFILE rows of
crates/signinum-j2k-cuda/src/runtime.rs:19-48 and SIGNINUM_J2K_PROFILE_STAGES
rows of crates/signinum-j2k-native/src/j2c/decode.rs:890-935).  Route rows
for the host branch and unsupported backends come before any CUDA call, so
they are checked here without a GPU; the stage rows of a device decode are
checked under the gpu mark."""
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent

CALLS = """
import ctypes
import numpy as np
from signinum_b200 import _native, encode
from signinum_b200._native import SgnRequest, SgnSurface
px = np.arange(16, dtype=np.uint8)
cs = encode.encode_lossless(px, 4, 4, 1, 8, levels=1, cb_exp=2, use_mct=False)
arr = np.frombuffer(cs, np.uint8)
lib = _native.cuda_lib()
out = SgnSurface()
for backend, kind in ((0, 0), (1, 1), (0, 1), (2, 0)):
    req = SgnRequest(kind, 0, 0, 2, 2, 1)
    lib.sgn_j2k_decode_to_device(None, arr.ctypes.data, arr.nbytes, 0, ctypes.byref(req), backend, ctypes.byref(out))
"""


def _run(env_value, code=CALLS, var="SIGNINUM_GPU_ROUTE_PROFILE"):
    env = dict(os.environ, PYTHONPATH=str(ROOT))
    env.pop("SIGNINUM_GPU_ROUTE_PROFILE", None)
    env.pop("SIGNINUM_J2K_PROFILE_STAGES", None)
    if env_value is not None:
        env[var] = env_value
    p = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    return [l for l in p.stderr.splitlines() if l.startswith("signinum_profile")]


@pytest.mark.parametrize("value", ["1", "TRUE", " yes ", "on", "Enabled"])
def test_route_rows_for_host_and_unsupported_backends(value):
    rows = _run(value)
    assert rows == [
        "signinum_profile codec=j2k op=gpu_route path=cuda op=full request=Auto fmt=Gray8 width=4 height=4 "
        "decision=host_surface",
        "signinum_profile codec=j2k op=gpu_route path=cuda op=region request=Cpu fmt=Gray8 width=4 height=4 "
        "decision=host_surface",
        "signinum_profile codec=j2k op=gpu_route path=cuda op=region request=Auto fmt=Gray8 width=4 height=4 "
        "decision=host_surface",
        "signinum_profile codec=j2k op=gpu_route path=cuda op=full request=Metal fmt=Gray8 width=4 height=4 "
        "decision=unsupported_backend",
    ]


def test_route_summary_counts_per_label_at_thread_exit():
    rows = _run("summary")
    assert sorted(rows) == sorted([
        "signinum_profile_summary codec=j2k op=gpu_route path=cuda route_op=full request=Auto fmt=Gray8 "
        "decision=host_surface count=1",
        "signinum_profile_summary codec=j2k op=gpu_route path=cuda route_op=full request=Metal fmt=Gray8 "
        "decision=unsupported_backend count=1",
        "signinum_profile_summary codec=j2k op=gpu_route path=cuda route_op=region request=Auto fmt=Gray8 "
        "decision=host_surface count=1",
        "signinum_profile_summary codec=j2k op=gpu_route path=cuda route_op=region request=Cpu fmt=Gray8 "
        "decision=host_surface count=1",
    ])


@pytest.mark.parametrize("value", [None, "", "0", "false", "off", "nope"])
def test_rows_off_unless_enabled(value):
    assert _run(value) == []


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["1", "summary"])
def test_stage_rows_of_a_device_decode(mode):
    code = """
from signinum_b200 import BackendRequest, Codec, J2kDecoder, PixelFormat, encode
w = encode.config2(n=6)
J2kDecoder(w.tiles[0].codestream).decode_to_device(PixelFormat.Rgb8, BackendRequest.Cuda)
Codec.decode_tiles_to_device([t.codestream for t in w.tiles], PixelFormat.Rgb8, BackendRequest.Cuda)
"""
    rows = _run(mode, code, "SIGNINUM_J2K_PROFILE_STAGES")
    if mode == "1":
        assert len(rows) == 2
        for row, tiles in zip(rows, (1, 6)):
            assert row.startswith("signinum_profile codec=j2k op=decode path=cuda tiles=%d " % tiles)
            f = dict(kv.split("=") for kv in row.split()[1:])
            for k in ("build_us", "ht_blocks", "ht_cleanup_bytes", "ht_vlc_us", "ht_mag_sgn_us", "idwt_us", "pack_us",
                      "total_us"):
                assert k in f, k
            assert int(f["ht_blocks"]) > 0 and int(f["ht_cleanup_bytes"]) > 0
            assert int(f["total_us"]) >= int(f["ht_cleanup_us"]) // 2
    else:
        assert len(rows) == 1
        f = dict(kv.split("=") for kv in rows[0].split()[1:])
        assert f["op"] == "decode" and f["count"] == "2"
        assert int(f["total_us_avg"]) == int(f["total_us_sum"]) // 2
        assert "ht_blocks_sum" in f and "ht_blocks_avg" not in f
