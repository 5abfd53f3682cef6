"""ctypes bindings of the package's native libraries.

The decode path lives in libsigninum_j2k_cuda.so (C ABI in
include/signinum_j2k_cuda.h); the encoder and synthetic tiles in
libsigninum_j2k_encode.so (include/signinum_j2k_encode.h).  There is no
fallback: a missing library raises at load time.
"""
import ctypes
import pathlib

LIB_DIR = pathlib.Path(__file__).resolve().parent / "_lib"
CUDA_LIB = LIB_DIR / "libsigninum_j2k_cuda.so"
ENCODE_LIB = LIB_DIR / "libsigninum_j2k_encode.so"

c_u8p = ctypes.POINTER(ctypes.c_uint8)


class SgnRequest(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_uint32), ("x", ctypes.c_uint32), ("y", ctypes.c_uint32),
                ("w", ctypes.c_uint32), ("h", ctypes.c_uint32), ("downscale", ctypes.c_uint32)]


class SgnSurface(ctypes.Structure):
    _fields_ = [("device_ptr", ctypes.c_uint64), ("width", ctypes.c_uint32), ("height", ctypes.c_uint32),
                ("format", ctypes.c_uint32), ("backend", ctypes.c_uint32), ("pitch_bytes", ctypes.c_uint64),
                ("kernel_dispatches", ctypes.c_uint64)]


class SgnInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in
                ("width", "height", "components", "bit_depth", "levels", "tiles", "ht", "reversible", "mct")]


class SgnHtBlock(ctypes.Structure):
    _fields_ = [("src", ctypes.c_uint64), ("dst", ctypes.c_uint64), ("reserved", ctypes.c_uint64),
                ("lcup", ctypes.c_uint32), ("tile", ctypes.c_uint32), ("stride", ctypes.c_uint32),
                ("lref", ctypes.c_uint16), ("w", ctypes.c_uint16), ("h", ctypes.c_uint16),
                ("missing_msbs", ctypes.c_uint8), ("passes", ctypes.c_uint8), ("num_bitplanes", ctypes.c_uint8),
                ("flags", ctypes.c_uint8), ("pad", ctypes.c_uint8 * 2)]


class SgnEncodeOptions(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in
                ("max_decomposition_levels", "code_block_width_exp", "code_block_height_exp", "use_mct",
                 "progression", "write_tlm", "sop_eph", "precinct_width_exp", "precinct_height_exp", "tile_parts")]


class SgnServerConfig(ctypes.Structure):
    _fields_ = [("device_budget_bytes", ctypes.c_uint64), ("resident_capacity_bytes", ctypes.c_uint64),
                ("max_batch_tiles", ctypes.c_uint32), ("slots", ctypes.c_uint32), ("reserved", ctypes.c_uint32),
                ("max_batch_samples", ctypes.c_uint64)]


class SgnServerResult(ctypes.Structure):
    _fields_ = [("ticket", ctypes.c_uint64), ("status", ctypes.c_int32), ("batch_tiles", ctypes.c_uint32),
                ("surface", SgnSurface), ("latency_ms", ctypes.c_double), ("queue_ms", ctypes.c_double)]


class SgnServerStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ("submitted", "completed", "batches", "rejected", "bytes_in_use",
                                               "peak_bytes_in_use")] + \
               [("max_batch_seen", ctypes.c_uint32), ("max_inflight_seen", ctypes.c_uint32),
                ("build_us_total", ctypes.c_uint64), ("gpu_us_total", ctypes.c_uint64),
                ("flight_us_total", ctypes.c_uint64)]


class SgnTuneReport(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ("vlc_threads", "ms_warps", "ms_blocks_per_grab", "dwt_queue")] + \
               [(n, ctypes.c_float) for n in ("vlc_ms", "ms_ms", "dwt_ms", "vlc_ms_default", "ms_ms_default",
                                              "dwt_ms_default")] + \
               [(n, ctypes.c_int32) for n in ("idwt_seg_shift", "pack_seg_shift")] + \
               [(n, ctypes.c_uint32) for n in ("vlc_lanes", "vlc_outline", "ht_fused")] + [("fused_ms", ctypes.c_float)] + \
               [("idwt_lean", ctypes.c_uint32)]


# Every entry point of include/signinum_j2k_cuda.h with its ctypes signature.
CUDA_SIGNATURES = {
    "sgn_dicom_frames": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_void_p,
                                          ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint64),
                                          ctypes.POINTER(ctypes.c_uint64), ctypes.c_size_t,
                                          ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]),
    "sgn_plan_set_launch_shape": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                                   ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]),
    "sgn_plan_autotune": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                           ctypes.POINTER(SgnTuneReport)]),
    "sgn_server_create": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(SgnServerConfig),
                                           ctypes.POINTER(ctypes.c_void_p)]),
    "sgn_server_register": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                             ctypes.POINTER(ctypes.c_uint32)]),
    "sgn_server_submit": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32,
                                           ctypes.POINTER(SgnRequest), ctypes.POINTER(ctypes.c_uint64)]),
    "sgn_server_submit_many": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint32),
                                                ctypes.c_uint32, ctypes.POINTER(SgnRequest),
                                                ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_size_t)]),
    "sgn_server_poll": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(SgnServerResult), ctypes.c_size_t,
                                         ctypes.POINTER(ctypes.c_size_t), ctypes.c_uint32]),
    "sgn_server_stats_get": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(SgnServerStats)]),
    "sgn_server_surface_free": (None, [ctypes.c_void_p, ctypes.POINTER(SgnSurface)]),
    "sgn_server_results_release": (None, [ctypes.c_void_p, ctypes.POINTER(SgnServerResult), ctypes.c_size_t]),
    "sgn_server_destroy": (None, [ctypes.c_void_p]),
    "sgn_ctx_create": (ctypes.c_int32, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "sgn_ctx_destroy": (None, [ctypes.c_void_p]),
    "sgn_ctx_submissions": (ctypes.c_uint64, [ctypes.c_void_p]),
    "sgn_last_error_message": (ctypes.c_char_p, []),
    "sgn_j2k_inspect": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(SgnInfo)]),
    "sgn_j2k_decode_to_device": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32,
                                                  ctypes.POINTER(SgnRequest), ctypes.c_uint32,
                                                  ctypes.POINTER(SgnSurface)]),
    "sgn_j2k_decode_tiles_to_device": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                                                        ctypes.POINTER(ctypes.c_size_t), ctypes.c_size_t,
                                                        ctypes.c_uint32, ctypes.POINTER(SgnRequest), ctypes.c_uint32,
                                                        ctypes.POINTER(SgnSurface), ctypes.POINTER(ctypes.c_int32),
                                                        ctypes.POINTER(ctypes.c_size_t)]),
    "sgn_surface_download": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(SgnSurface), ctypes.c_void_p,
                                              ctypes.c_size_t, ctypes.c_size_t]),
    "sgn_surface_free": (None, [ctypes.c_void_p, ctypes.POINTER(SgnSurface)]),
    "sgn_plan_create": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                                         ctypes.POINTER(ctypes.c_size_t), ctypes.c_size_t, ctypes.c_uint32,
                                         ctypes.POINTER(SgnRequest), ctypes.POINTER(ctypes.c_void_p),
                                         ctypes.POINTER(ctypes.c_int32)]),
    "sgn_plan_execute_async": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p]),
    "sgn_plan_wait": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32),
                                       ctypes.POINTER(ctypes.c_size_t)]),
    "sgn_plan_surfaces": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(SgnSurface), ctypes.c_size_t]),
    "sgn_plan_kernel_launches": (ctypes.c_uint64, [ctypes.c_void_p]),
    "sgn_plan_execute_timed": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)]),
    "sgn_plan_destroy": (None, [ctypes.c_void_p, ctypes.c_void_p]),
    "sgn_ctx_stream": (ctypes.c_void_p, [ctypes.c_void_p]),
    "sgn_ht_lookup_tables": (None, [ctypes.c_void_p] * 4),
    "sgn_ebcot_tables": (None, [ctypes.c_void_p] * 6),
    "sgn_j2k_ht_block_table": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t,
                                                ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_uint64)]),
    "sgn_plan_tile_coefficients": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                                    ctypes.c_void_p, ctypes.c_size_t,
                                                    ctypes.POINTER(ctypes.c_size_t)]),
    "sgn_j2k_request_blocks": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32,
                                                ctypes.POINTER(SgnRequest), ctypes.POINTER(ctypes.c_uint64),
                                                ctypes.POINTER(ctypes.c_uint64)]),
    "sgn_plan_set_tile_shape": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32]),
    "sgn_plan_set_cleanup_form": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32]),
    "sgn_ht_decode_blocks_noalloc": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                                      ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t,
                                                      ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p]),
}

ENCODE_SIGNATURES = {
    "sgn_j2k_encode_lossless": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                               ctypes.c_uint32, ctypes.POINTER(SgnEncodeOptions), ctypes.c_void_p,
                                               ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "sgn_j2k_encode_irreversible": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                                   ctypes.c_uint32, ctypes.POINTER(SgnEncodeOptions), ctypes.c_double,
                                                   ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "sgn_j2k_encode_classic": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                              ctypes.c_uint32, ctypes.POINTER(SgnEncodeOptions), ctypes.c_uint32,
                                              ctypes.c_uint32, ctypes.c_double, ctypes.c_uint32, ctypes.c_void_p,
                                              ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "sgn_synth_he_rgb8": (None, [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_double, ctypes.c_void_p]),
    "sgn_synth_blank_rgb8": (None, [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p]),
    "sgn_synth_fluor_gray16": (None, [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p]),
}

_cuda = None
_encode = None


def _bind(path, sigs):
    if not path.exists():
        raise RuntimeError(f"native library {path.name} is not built; run `python -m signinum_b200.build`")
    lib = ctypes.CDLL(str(path))
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def cuda_lib():
    global _cuda
    if _cuda is None:
        _cuda = _bind(CUDA_LIB, CUDA_SIGNATURES)
    return _cuda


def encode_lib():
    global _encode
    if _encode is None:
        _encode = _bind(ENCODE_LIB, ENCODE_SIGNATURES)
    return _encode


def last_error():
    msg = cuda_lib().sgn_last_error_message()
    return msg.decode() if msg else ""
