"""Builds the native libraries of the package in-tree.

    python -m signinum_b200.build          # or signinum_b200.build.build_all()

libsigninum_j2k_cuda.so    the sm_100a decode path and its C ABI
                           (include/signinum_j2k_cuda.h)
libsigninum_j2k_encode.so  the lossless HTJ2K encoder and synthetic tiles
                           (include/signinum_j2k_encode.h)

Compiled with nvcc for sm_100a only (-gencode arch=compute_100a,code=sm_100a).
Outputs go to signinum_b200/_lib/ so they travel with the source tree.
"""
import os
import pathlib
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = PKG / "_lib"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CUDA_SOURCES = [
    CSRC / "kernels" / "ht_decode.cu",
    CSRC / "kernels" / "idwt_pack.cu",
    CSRC / "kernels" / "classic_decode.cu",
    CSRC / "host" / "runtime.cu",
    CSRC / "host" / "noalloc.cu",
    CSRC / "host" / "server.cu",
    CSRC / "host" / "dicom.cpp",
    CSRC / "host" / "codestream.cpp",
]
ENCODE_SOURCES = [
    CSRC / "encode" / "j2k_encode.cpp",
    CSRC / "encode" / "classic_encode.cpp",
    CSRC / "encode" / "synth.cpp",
    CSRC / "encode" / "encode_capi.cpp",
]


def _deps():
    files = list(CSRC.rglob("*")) + list((ROOT / "include").glob("*.h"))
    return [f for f in files if f.is_file()]


def _stale(target, deps):
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd):
    print(" ".join(str(c) for c in cmd), flush=True)
    subprocess.run([str(c) for c in cmd], check=True)


def build_cuda(force=False):
    target = OUT / "libsigninum_j2k_cuda.so"
    if not force and not _stale(target, _deps()):
        return target
    OUT.mkdir(exist_ok=True)
    cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "--use_fast_math", "-Xcompiler", "-fPIC,-O3",
           "-shared", "-o", target, "-I", ROOT / "include", *CUDA_SOURCES]
    # --use_fast_math is not wanted for the pack conversions: they call the
    # IEEE intrinsics (__fdiv_rn, __fmul_rn) explicitly, and no other float
    # arithmetic runs on the path.
    cmd.remove("--use_fast_math")
    _run(cmd)
    return target


def build_encoder(force=False):
    target = OUT / "libsigninum_j2k_encode.so"
    if not force and not _stale(target, _deps()):
        return target
    OUT.mkdir(exist_ok=True)
    _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", target, "-I", ROOT / "include", *ENCODE_SOURCES])
    return target


def build_all(force=False):
    return build_cuda(force), build_encoder(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
