/* signinum-j2k-cuda drop-in: HTJ2K tile decode into CUDA device memory (sm_100a).
 *
 * C ABI of the decode path behind the reference's CUDA adapter
 * (crates/signinum-j2k-cuda, frames-sg/signinum 0.4.2).  Every entry point
 * names the reference interface it replaces.  Plain pointers and sizes only;
 * device memory is this library's own (CUDA runtime, device chosen at
 * context creation).
 *
 * Status codes map one to one onto the reference's Error variants and
 * predicates (crates/signinum-j2k-cuda/src/error.rs:7-41):
 *   SGN_ERR_UNSUPPORTED / SGN_ERR_UNSUPPORTED_BACKEND / SGN_ERR_CUDA_UNAVAILABLE
 *       -> is_unsupported();   SGN_ERR_BUFFER -> is_buffer_error();
 *   SGN_ERR_TRUNCATED -> is_truncated();  SGN_ERR_REGION -> J2kError::InvalidRegion;
 *   SGN_ERR_DECODE -> other decode errors;  SGN_ERR_CUDA_RUNTIME -> CudaRuntime{message};
 *   SGN_ERR_HOST_BACKEND -> not an error in the reference: the adapter's host
 *       branch for BackendRequest::Cpu / ::Auto, which this library leaves
 *       to the caller.
 */
#ifndef SIGNINUM_J2K_CUDA_H
#define SIGNINUM_J2K_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t sgn_status;
enum {
  SGN_OK = 0,
  SGN_ERR_UNSUPPORTED = 1,
  SGN_ERR_BUFFER = 2,
  SGN_ERR_TRUNCATED = 3,
  SGN_ERR_DECODE = 4,
  SGN_ERR_REGION = 5,
  SGN_ERR_CUDA_UNAVAILABLE = 6,
  SGN_ERR_CUDA_RUNTIME = 7,
  SGN_ERR_UNSUPPORTED_BACKEND = 8,
  SGN_ERR_INVALID_ARGUMENT = 9,
  SGN_ERR_OUT_OF_MEMORY = 10,
  /* BackendRequest::Cpu or ::Auto: the request belongs to the adapter's host
   * branch (wrap_surface returns a host Surface of the CPU decoder's bytes,
   * crates/signinum-j2k-cuda/src/runtime.rs:19-48).  Returned before any
   * CUDA call; no context is needed or created. */
  SGN_ERR_HOST_BACKEND = 11
};

/* signinum_core::PixelFormat (crates/signinum-core/src/types.rs). */
typedef enum sgn_pixel_format {
  SGN_FMT_GRAY8 = 0,
  SGN_FMT_RGB8 = 1,
  SGN_FMT_RGBA8 = 2,
  SGN_FMT_GRAY16 = 3,
  SGN_FMT_RGB16 = 4,
  SGN_FMT_RGBA16 = 5 /* rejected as unsupported, as the reference does (decode.rs:358-366) */
} sgn_pixel_format;

/* signinum_core::BackendRequest (crates/signinum-core/src/backend.rs:15-22).
 * Only CUDA decodes here.  CPU and AUTO return SGN_ERR_HOST_BACKEND before
 * any CUDA call: the reference serves both with a host surface and never
 * initialises CUDA for them (runtime.rs:19-48, session.rs:32-38), so the
 * adapter keeps that branch and routes only CUDA to this library.  METAL is
 * SGN_ERR_UNSUPPORTED_BACKEND (validate_surface_request, runtime.rs:52-57). */
typedef enum sgn_backend_request {
  SGN_BACKEND_AUTO = 0,
  SGN_BACKEND_CPU = 1,
  SGN_BACKEND_METAL = 2,
  SGN_BACKEND_CUDA = 3
} sgn_backend_request;

/* DeviceDecodeRequest (crates/signinum-j2k/src/adapter/device_plan.rs:7-12);
 * downscale is the Downscale denominator 1, 2, 4 or 8
 * (crates/signinum-core/src/scale.rs:5-20). */
typedef enum sgn_request_kind {
  SGN_REQ_FULL = 0,
  SGN_REQ_REGION = 1,
  SGN_REQ_SCALED = 2,
  SGN_REQ_REGION_SCALED = 3
} sgn_request_kind;

typedef struct sgn_request {
  uint32_t kind; /* sgn_request_kind */
  uint32_t x, y, w, h;
  uint32_t downscale;
} sgn_request;

/* Surface + CudaSurface (crates/signinum-j2k-cuda/src/surface.rs:19-127):
 * tight rows, pitch_bytes = width * bytes_per_pixel. */
typedef struct sgn_surface {
  uint64_t device_ptr;
  uint32_t width, height;
  uint32_t format;           /* sgn_pixel_format */
  uint32_t backend;          /* always SGN_BACKEND_CUDA for a decoded surface */
  uint64_t pitch_bytes;
  uint64_t kernel_dispatches; /* CudaSurfaceStats::kernel_dispatches */
} sgn_surface;

/* J2kView::inspect info (crates/signinum-core/src/types.rs Info). */
typedef struct sgn_info {
  uint32_t width, height, components, bit_depth, levels, tiles, ht, reversible, mct;
} sgn_info;

typedef struct sgn_ctx sgn_ctx;

/* Replaces CudaSession + CudaContext::system_default
 * (crates/signinum-j2k-cuda/src/session.rs:11-39,
 * crates/signinum-cuda-runtime/src/lib.rs:286-320). */
sgn_status sgn_ctx_create(int device, sgn_ctx** out);
void sgn_ctx_destroy(sgn_ctx* ctx);
/* CudaSession::submissions (session.rs:19-21). */
uint64_t sgn_ctx_submissions(const sgn_ctx* ctx);
/* Message of the last failing call on this thread. */
const char* sgn_last_error_message(void);

/* J2kDecoder::inspect / J2kView::parse (crates/signinum-j2k/src/view.rs:42-58). */
sgn_status sgn_j2k_inspect(const uint8_t* data, size_t len, sgn_info* out);

/* The plain per-tile drop-in: J2kDecoder::{decode,decode_region,decode_scaled,
 * decode_region_scaled}_to_device (crates/signinum-j2k-cuda/src/decoder.rs:31-140)
 * and Codec::submit_tile*_to_device (codec.rs:27-188).  Synchronous; on success
 * *out owns a device buffer released by sgn_surface_free. */
sgn_status sgn_j2k_decode_to_device(sgn_ctx* ctx, const uint8_t* data, size_t len, uint32_t format,
                                    const sgn_request* request, uint32_t backend, sgn_surface* out);

/* The batched form: TileBatchDecodeManyDevice::decode_tiles_to_device
 * (crates/signinum-j2k-cuda/src/codec.rs:190-209).  One request per tile
 * (NULL = full decode of every tile).  Order is preserved; per_tile[i] gets
 * each tile's status; *first_failing gets the lowest failing index or
 * SIZE_MAX, mirroring TileBatchError (crates/signinum-core/src/batch.rs:41-77).
 * Returns SGN_OK when every tile decoded, else the status of the first
 * failing tile; surfaces of successful tiles are valid either way. */
sgn_status sgn_j2k_decode_tiles_to_device(sgn_ctx* ctx, const uint8_t* const* datas, const size_t* lens, size_t n,
                                          uint32_t format, const sgn_request* requests, uint32_t backend,
                                          sgn_surface* outs, sgn_status* per_tile, size_t* first_failing);

/* Surface::download_into (surface.rs:78-92): tight device-to-host copy into
 * rows of `stride` bytes (stride >= pitch_bytes). */
sgn_status sgn_surface_download(sgn_ctx* ctx, const sgn_surface* surface, uint8_t* out, size_t out_len, size_t stride);
/* Releases the device buffer (CudaDeviceBuffer drop, crates/signinum-cuda-runtime/src/lib.rs:955-964). */
void sgn_surface_free(sgn_ctx* ctx, sgn_surface* surface);

/* ---- Device-resident batch plans (no counterpart in the reference: the
 * split of decode_tiles_to_device into host parse + device execute lets a
 * caller keep codestreams resident and replay decodes). */
typedef struct sgn_plan sgn_plan;
/* Parses the batch, uploads codestreams and descriptor tables, allocates the
 * output surfaces.  Per-tile parse failures are reported like
 * decode_tiles_to_device. */
sgn_status sgn_plan_create(sgn_ctx* ctx, const uint8_t* const* datas, const size_t* lens, size_t n, uint32_t format,
                           const sgn_request* requests, sgn_plan** out, sgn_status* per_tile);
/* Enqueues the kernels of the plan on the context stream (no host sync).
 * From the second execution on, the plan runs as one captured CUDA graph. */
sgn_status sgn_plan_execute_async(sgn_ctx* ctx, sgn_plan* plan);
/* Waits for the plan and gathers per-tile statuses. */
sgn_status sgn_plan_wait(sgn_ctx* ctx, sgn_plan* plan, sgn_status* per_tile, size_t* first_failing);
/* Surfaces of the plan (valid until sgn_plan_destroy). */
sgn_status sgn_plan_surfaces(const sgn_plan* plan, sgn_surface* outs, size_t n);
/* Executes the plan with CUDA events around each stage on the launching
 * stream and waits; stage_ms (6 entries) receives {HT cleanup VLC pass, HT
 * cleanup MagSgn pass, HT refinement, IDWT levels, last level + pack, total}
 * in milliseconds (no counterpart in the reference: measurement). */
sgn_status sgn_plan_execute_timed(sgn_ctx* ctx, sgn_plan* plan, float* stage_ms);
/* Autotuner (no counterpart in the reference).  Times the plan's stages on
 * its own data over `reps` runs each (0: 5) for every candidate launch shape
 * (VLC threads per CTA, code blocks per VLC warp and its bit-reader refills
 * inline or out of line; for plans of up to 8192 code blocks, both cleanup
 * passes fused in one kernel against the best separate pair; MagSgn warps per CTA, one block per warp or persistent
 * warps taking 1 or 4 blocks per grab from the device work queue; IDWT and
 * pack, each, one unit per warp (for IDWT also at four CTAs per SM) or persistent on a queue: dwt_queue bit 0 =
 * IDWT levels, bit 1 = pack; and the DWT tile shape of each, 128 columns by
 * the base rows per unit scaled by 2^shift, shift -4 to 1), keeps the fastest per
 * stage for the plan and for later plans of the same shape on this context,
 * and re-executes the plan so its surfaces hold the decode.  Synchronous. */
typedef struct sgn_tune_report {
  uint32_t vlc_threads, ms_warps, ms_blocks_per_grab, dwt_queue;  /* chosen shape */
  float vlc_ms, ms_ms, dwt_ms;                                     /* its stage times */
  float vlc_ms_default, ms_ms_default, dwt_ms_default;             /* the default shape's */
  int32_t idwt_seg_shift, pack_seg_shift;                          /* chosen DWT tile shape (rows x 2^shift) */
  uint32_t vlc_lanes;                                              /* chosen code blocks per VLC warp */
  uint32_t vlc_outline; /* 1: the VLC pass's bit-reader refills out of line, 0: inline */
  uint32_t ht_fused;    /* 1: both cleanup passes in one kernel, a CTA per code block (small plans) */
  float fused_ms;       /* that kernel's time (0: not tried) */
  uint32_t idwt_lean;   /* 1: the IDWT levels' grid form held to four CTAs per SM */
} sgn_tune_report;
sgn_status sgn_plan_autotune(sgn_ctx* ctx, sgn_plan* plan, uint32_t reps, sgn_tune_report* out);
/* Sets the launch shape by hand (the fields of sgn_tune_report's first row;
 * vlc_threads 32..128 in steps of 32, ms_warps 1..8, dwt_queue 0..3). */
sgn_status sgn_plan_set_launch_shape(sgn_ctx* ctx, sgn_plan* plan, uint32_t vlc_threads, uint32_t ms_warps,
                                     uint32_t ms_blocks_per_grab, uint32_t dwt_queue);
/* Sets the DWT tile shape by hand: rows per work unit of the IDWT levels and
 * of the last level + pack, the base rule scaled by 2^shift (shift -4 to 1;
 * strips stay 128 columns wide).  Re-uploads the plan's job tables. */
sgn_status sgn_plan_set_tile_shape(sgn_ctx* ctx, sgn_plan* plan, int32_t idwt_seg_shift, int32_t pack_seg_shift);
/* Sets the HT cleanup form by hand (no counterpart in the reference): 0, the
 * VLC pass then the MagSgn pass over all blocks; 1, both passes of each block
 * in one CTA, its MagSgn following its VLC chain row by row (the default for
 * plans of few blocks); 2, chosen by block count.  Decodes are the same. */
sgn_status sgn_plan_set_cleanup_form(sgn_ctx* ctx, sgn_plan* plan, uint32_t fused);
/* Launches issued by one execute of the plan. */
uint64_t sgn_plan_kernel_launches(const sgn_plan* plan);
void sgn_plan_destroy(sgn_ctx* ctx, sgn_plan* plan);
/* The context's CUDA stream (cudaStream_t) for event timing by callers. */
void* sgn_ctx_stream(sgn_ctx* ctx);

/* Diagnostics (no counterpart in the reference): copies the packed HT lookup
 * tables the kernels decode with (VLC initial/other rows: 1024 entries each;
 * UVLC initial row: 320; other rows: 256) so tests can pin them to the
 * reference's ht_tables.rs. */
void sgn_ht_lookup_tables(uint16_t* vlc0, uint16_t* vlc1, uint16_t* uvlc0, uint16_t* uvlc1);

/* Diagnostics (no counterpart in the reference): the classic Tier-1 tables
 * the kernels decode with, as the reference lays them out: zero-coding
 * contexts for LL/LH, HL and HH bands and the sign-coding (label, xor)
 * pairs, 256 entries each over the neighbour-significance byte, and the MQ
 * probability table as 47 little-endian (u16 qe, u8 nmps, u8 nlps,
 * u8 switch) records (235 bytes), so tests can pin them to the reference. */
void sgn_ebcot_tables(uint8_t* zc_ll_lh, uint8_t* zc_hl, uint8_t* zc_hh, uint8_t* sc_label, uint8_t* sc_xor,
                      uint8_t* qe_records);

/* One HT code block for the block-level entry points below: where its
 * cleanup segment starts in a segment buffer (the refinement segment, if
 * any, follows it), where its first sample goes in an int32 coefficient
 * buffer and how rows are strided there. */
typedef struct sgn_ht_block {
  uint64_t src;           /* byte offset of the cleanup segment */
  uint64_t dst;           /* element offset of sample (0, 0) */
  uint64_t reserved;      /* filled by the library */
  uint32_t lcup;          /* cleanup segment length */
  uint32_t tile;          /* index into the status array */
  uint32_t stride;        /* row stride in elements */
  uint16_t lref;          /* refinement segment length */
  uint16_t w, h;          /* block size, at most 4096 samples */
  uint8_t missing_msbs;   /* missing MSBs after placeholder passes are folded in */
  uint8_t passes;         /* 0 = all-zero block, 1 cleanup, 2 + SigProp, 3 + MagRef */
  uint8_t num_bitplanes;  /* magnitude bit-planes of the band */
  uint8_t flags;          /* bit 0: vertically causal context */
  uint8_t pad[2];
} sgn_ht_block;

/* Diagnostics (no counterpart in the reference): the code-block table of a
 * full-resolution decode of one codestream, as the decode path builds it,
 * with src relative to the codestream and dst into one tight int32 buffer of
 * *coef_elems elements (per component: LL, then HL/LH/HH per resolution).
 * *count receives the number of blocks (also when cap is too small:
 * SGN_ERR_BUFFER). */
sgn_status sgn_j2k_ht_block_table(const uint8_t* data, size_t len, sgn_ht_block* out, size_t cap, size_t* count,
                                  uint64_t* coef_elems);
/* Diagnostics (no counterpart in the reference's interface; host only, no
 * CUDA): the code blocks a decode of `request` (NULL: full image) at pixel
 * format `format` decodes (*decoded) out of the blocks of the decoded
 * resolutions (*total).  Region requests decode only the blocks their region
 * needs (RoiPlan::code_block_required,
 * crates/signinum-j2k-native/src/j2c/roi.rs:108-113); other requests all. */
sgn_status sgn_j2k_request_blocks(const uint8_t* data, size_t len, uint32_t format, const sgn_request* request,
                                  uint64_t* decoded, uint64_t* total);
/* Diagnostics: copies tile `tile`'s sub-band coefficients (the HT stage
 * output, same layout as sgn_j2k_ht_block_table) of an executed plan to host
 * memory; *count receives the element count. */
sgn_status sgn_plan_tile_coefficients(sgn_ctx* ctx, const sgn_plan* plan, size_t tile, int32_t* out, size_t cap,
                                      size_t* count);

/* HT code-block decode that allocates nothing (no counterpart in the
 * reference: its adapter has no block-level entry point).
 *
 * For callers of this code that cannot allocate device memory: a host
 * framework whose caching allocator owns all of the GPU's memory (a
 * cudaMalloc beside it fails or fragments that pool), a decoder plugin that
 * is handed its input and output buffers by its host and may create none of
 * its own, and real-time loops that must not allocate, nor wait on the
 * allocator's implicit synchronisation, once they run.  The caller passes
 * device memory for the inputs (`segments`, segments_len bytes, the buffer
 * the blocks' src offsets point into) and the outputs (`coefficients`,
 * coefficients_len int32 elements, 8-byte aligned; `tile_status`, n_tiles
 * words, set to nonzero for tiles with a block that failed to decode);
 * `blocks` is a host array.  Every block's reads must lie inside
 * segments[0, segments_len) and its writes inside
 * coefficients[0, coefficients_len), else the call returns SGN_ERR_BUFFER
 * before any device work.
 *
 * The scratch the HT kernels need lives in fixed static device arrays
 * (16 MiB of quad symbols plus the device copy of the block table, about
 * 16.4 MiB in all): at most 4096 blocks of at most 4096 samples per call,
 * cleanup segments up to about 27 KB; larger requests are rejected with
 * SGN_ERR_INVALID_ARGUMENT or SGN_ERR_UNSUPPORTED before any device work.
 * The arrays stay reserved on every device where the library's module that
 * holds them is loaded (with CUDA's default lazy loading: from this entry
 * point's first call on that device) until the process exits.
 *
 * Runs asynchronously on `stream` (a cudaStream_t; NULL = the legacy default
 * stream) on the current device.  The first call on a device does the
 * per-device set-up (it looks up the static arrays' device addresses with
 * cudaGetSymbolAddress); make that first call before any stream capture.
 * All calls on a device share the static arrays and leave the last call's
 * contents there: calls that overlap on the GPU race and must be serialised
 * by the caller.  tile_status is cleared by the call. */
sgn_status sgn_ht_decode_blocks_noalloc(const sgn_ht_block* blocks, uint32_t n, const uint8_t* segments,
                                        size_t segments_len, int32_t* coefficients, size_t coefficients_len,
                                        uint32_t* tile_status, uint32_t n_tiles, void* stream);

/* ---- DICOM input: extract_dicom_encapsulated_frames_with_limit
 * (crates/signinum-j2k-metal/src/dicom.rs:22-95).  Extracts up to `limit`
 * frames (SIZE_MAX: all) of the encapsulated Pixel Data of a DICOM file:
 * grouped by the Basic Offset Table, else by the Extended Offset Table (its
 * Lengths trim padded frames), else one frame per fragment.  Call once with
 * out == NULL for *nframes and *out_bytes, then with buffers of that size:
 * the frames are written back to back into `out`, each 16-byte aligned, at
 * frame_offsets[i] with frame_lens[i] bytes, ready for
 * sgn_j2k_decode_tiles_to_device.  Errors: SGN_ERR_TRUNCATED, SGN_ERR_DECODE
 * (malformed / no Pixel Data), SGN_ERR_UNSUPPORTED (native Pixel Data),
 * SGN_ERR_BUFFER (buffers too small).  Host only. */
sgn_status sgn_dicom_frames(const uint8_t* data, size_t len, size_t limit, uint8_t* out, size_t out_cap,
                            uint64_t* frame_offsets, uint64_t* frame_lens, size_t frames_cap, size_t* nframes,
                            size_t* out_bytes);

/* ---- Serving loop: continuous batching of tile requests (sgn_server_submit /
 * sgn_server_poll stand beside the drop-in calls; the reference has no
 * serving loop, its adapter decodes one call at a time).
 *
 * Codestreams are registered once and stay resident in device memory.
 * Requests (full, region, reduced resolution, region at reduced resolution,
 * any pixel format the plain call accepts) are queued as they arrive; a
 * dispatcher thread forms a batch from the queue whenever one of `slots`
 * CUDA streams is free and the batch's estimated device memory fits in
 * `device_budget_bytes` beside the batches already on the GPU, so requests
 * that arrive while others decode are admitted as slots and memory free up
 * and their work overlaps on the device.  A completion thread publishes each
 * request's surface, status and latency (submit to publication, host clock)
 * as its batch finishes. */
typedef struct sgn_server sgn_server;

typedef struct sgn_server_config {
  uint64_t device_budget_bytes;     /* admission budget for in-flight batches (0: 16 GiB) */
  uint64_t resident_capacity_bytes; /* device arena for registered codestreams (0: 1 GiB) */
  uint32_t max_batch_tiles;         /* requests per batch (0: 512) */
  uint32_t slots;                   /* batches in flight at once, one CUDA stream each (0: 3) */
  uint32_t reserved;
  uint64_t max_batch_samples;       /* decoded samples per batch, bounds a batch's GPU time (0: no bound) */
} sgn_server_config;

typedef struct sgn_server_result {
  uint64_t ticket;
  sgn_status status;       /* per request, as sgn_j2k_decode_to_device reports it */
  uint32_t batch_tiles;    /* requests in the batch that carried this one */
  sgn_surface surface;     /* owned by the caller when status is SGN_OK: sgn_server_surface_free */
  double latency_ms;       /* submit -> result published */
  double queue_ms;         /* submit -> batch launched */
} sgn_server_result;

typedef struct sgn_server_stats {
  uint64_t submitted, completed, batches, rejected;
  uint64_t bytes_in_use, peak_bytes_in_use;
  uint32_t max_batch_seen, max_inflight_seen;
  uint64_t build_us_total;  /* dispatcher time spent building and launching batches */
  uint64_t gpu_us_total;    /* device time of the batches' kernels (CUDA events) */
  uint64_t flight_us_total; /* batch launched -> batch results published */
} sgn_server_stats;

sgn_status sgn_server_create(sgn_ctx* ctx, const sgn_server_config* config, sgn_server** out);
/* Copies a codestream into the resident arena; *tile_id names it in requests. */
sgn_status sgn_server_register(sgn_server* server, const uint8_t* data, size_t len, uint32_t* tile_id);
/* Queues a request (request NULL = full image); validation that needs no
 * parse (format, request kind, region bounds, budget) fails here. */
sgn_status sgn_server_submit(sgn_server* server, uint32_t tile_id, uint32_t format, const sgn_request* request,
                             uint64_t* ticket);
/* Queues n requests in one call (requests NULL = all full images), in order;
 * stops at the first invalid one and returns its status, *submitted telling
 * how many went in. */
sgn_status sgn_server_submit_many(sgn_server* server, size_t n, const uint32_t* tile_ids, uint32_t format,
                                  const sgn_request* requests, uint64_t* tickets, size_t* submitted);
/* Moves up to cap published results into out (*count of them), waiting up to
 * timeout_ms for the first one (0: no wait). */
sgn_status sgn_server_poll(sgn_server* server, sgn_server_result* out, size_t cap, size_t* count, uint32_t timeout_ms);
sgn_status sgn_server_stats_get(sgn_server* server, sgn_server_stats* out);
/* Frees a result surface without synchronising the device. */
void sgn_server_surface_free(sgn_server* server, sgn_surface* surface);
/* Frees the surfaces of n polled results at once (entries already freed or
 * failed are skipped). */
void sgn_server_results_release(sgn_server* server, sgn_server_result* results, size_t n);
/* Finishes every queued and in-flight request, then releases the server;
 * results not yet polled are freed. */
void sgn_server_destroy(sgn_server* server);

#ifdef __cplusplus
}
#endif

#endif
