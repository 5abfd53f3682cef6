"""signinum_b200: B200-native HTJ2K tile decode into CUDA device memory.

A from-scratch sm_100a implementation of frames-sg/signinum's HTJ2K
tile-batch decode path, behind a C ABI (include/signinum_j2k_cuda.h) that
mirrors the reference's signinum-j2k-cuda adapter; j2k_cuda is its Python
face.
"""
from .j2k_cuda import (BackendKind, BackendRequest, Codec, CudaSession, CudaSurface, Downscale, Error, J2kDecoder,
                       PixelFormat, Rect, Surface, TileBatchError, dicom_frames, inspect, set_host_decoder)

__all__ = ["BackendKind", "BackendRequest", "Codec", "CudaSession", "CudaSurface", "Downscale", "Error",
           "J2kDecoder", "PixelFormat", "Rect", "Surface", "TileBatchError", "dicom_frames", "inspect",
           "set_host_decoder"]
