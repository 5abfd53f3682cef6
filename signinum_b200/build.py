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
    CSRC / "host" / "profile.cpp",
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
    """Compiles every source to an object in parallel, then links the
    library.  No --use_fast_math: the pack conversions call the IEEE
    intrinsics (__fdiv_rn, __fmul_rn) explicitly and nothing else on the
    path needs it."""
    from concurrent.futures import ThreadPoolExecutor

    target = OUT / "libsigninum_j2k_cuda.so"
    deps = _deps()
    if not force and not _stale(target, deps):
        return target
    objdir = OUT / "obj"
    objdir.mkdir(parents=True, exist_ok=True)
    common = [*ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "-I", ROOT / "include"]

    def compile_one(src):
        obj = objdir / (src.stem + src.suffix.replace(".", "_") + ".o")
        if force or _stale(obj, deps):
            _run([NVCC, *common, "-c", "-o", obj, src])
        return obj

    with ThreadPoolExecutor(max_workers=len(CUDA_SOURCES)) as ex:
        objs = list(ex.map(compile_one, CUDA_SOURCES))
    tmp = target.with_suffix(".so.tmp")
    _run([NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", tmp, *objs])
    os.replace(tmp, target)  # a reader never sees a half-written library
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
