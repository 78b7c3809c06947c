/*
 * wgpufft_b200 — C ABI of the B200 (sm_100a) FFT transform path.
 *
 * Drop-in boundary for the public plan API of the Rust crate wgpu-fft
 * (MaximEremenko/wgpuFFT): every entry point below names the crate function
 * it replaces (file:line in that project).  wgpu handles become CUDA ones:
 * a `wgpu::Buffer` becomes a device pointer plus its size in bytes, a
 * `wgpu::CommandEncoder` becomes a CUDA stream (`cudaStream_t` passed as
 * `void*`; NULL is the legacy default stream), and `queue.submit` becomes the
 * stream's own ordering.  Plans record work onto the caller's stream and
 * return without synchronising, as the crate's plans record into the
 * caller's encoder (src/plan.rs:494-518).
 *
 * Layout conventions are the crate's: interleaved complex values
 * ([re, im] for f32/f64, [re_hi, re_lo, im_hi, im_lo] f32 words for df64),
 * axis 0 contiguous, batches as contiguous blocks, real transforms' packed
 * spectrum [N0/2 + 1, N1, ...] (README.md:111-128, src/math/mod.rs:444-448).
 *
 * Errors: every fallible call returns a b2f_status whose values mirror the
 * crate's FftError variants (src/error.rs:12-177); b2f_last_error_message()
 * gives the detail of the calling thread's last failure.  Nothing panics or
 * throws across the ABI.
 *
 * Threading: a plan is immutable after creation and may be executed from
 * several threads on different streams at once.  A plan whose executions
 * share device memory (a multi-pass route's workspace, the in-place copy
 * buffer of a real transform, created on first use under a lock) orders
 * them on the device itself: each execution waits for the previous one's
 * completion event and records its own, so executions on different streams
 * run one after the other instead of racing.  Executions recorded into a
 * CUDA graph (b2f_plan_record, or any stream capture) skip that event pair;
 * the graph's own order applies, and a graph launched concurrently with an
 * eager execution of the same plan must be ordered by the caller.  A batch
 * (b2f_batch_*) keeps its work-queue counters and internal streams per
 * object: executions of one batch must be ordered by the caller (one
 * stream, or events).
 */
#ifndef WGPUFFT_B200_H
#define WGPUFFT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t b2f_status;

/* Status codes (src/error.rs:12-177 variant in brackets). */
#define B2F_OK 0
#define B2F_ERR_ZERO_LENGTH 1              /* FftError::ZeroLength */
#define B2F_ERR_ZERO_BATCH 2               /* FftError::ZeroBatch */
#define B2F_ERR_LENGTH_TOO_LARGE 3         /* FftError::LengthTooLarge */
#define B2F_ERR_UNSUPPORTED_LENGTH 4       /* FftError::UnsupportedLength */
#define B2F_ERR_PRECISION_UNSUPPORTED 5    /* FftError::PrecisionUnsupported */
#define B2F_ERR_INVALID_TUNING 6           /* FftError::InvalidTuning */
#define B2F_ERR_EMPTY_AXES 7               /* FftError::EmptyAxes */
#define B2F_ERR_INVALID_AXIS 8             /* FftError::InvalidAxis */
#define B2F_ERR_DUPLICATE_AXIS 9           /* FftError::DuplicateAxis */
#define B2F_ERR_INVALID_REAL_DIRECTION 10  /* FftError::InvalidRealTransformDirection */
#define B2F_ERR_UNSUPPORTED_REAL_AXES 11   /* FftError::UnsupportedRealAxes */
#define B2F_ERR_BUFFER_TOO_SMALL 12        /* FftError::BufferViewTooSmall */
#define B2F_ERR_IN_PLACE_UNSUPPORTED 13    /* FftError::InPlaceUnsupported */
#define B2F_ERR_RESOURCE_ALLOCATION 14     /* FftError::GpuPlanResourceAllocationFailed */
#define B2F_ERR_INVALID_ARGUMENT 15        /* null handle or pointer (Rust references cannot be null) */
#define B2F_ERR_DEVICE 16                  /* a CUDA call failed (wgpu validation/device error) */
#define B2F_ERR_WORKSPACE_TOO_SMALL 17     /* FftError::WorkspaceTooSmall */
/* Tuning-snapshot decoding, the four variants of the crate's
 * PipelineCacheSnapshotError (src/runtime/pipeline_cache.rs:58-74). */
#define B2F_ERR_SNAPSHOT_JSON 18           /* PipelineCacheSnapshotError::Json */
#define B2F_ERR_SNAPSHOT_SCHEMA 19         /* PipelineCacheSnapshotError::SchemaMismatch */
#define B2F_ERR_SNAPSHOT_VERSION 20        /* PipelineCacheSnapshotError::VersionMismatch */
#define B2F_ERR_SNAPSHOT_INTEGRITY 21      /* PipelineCacheSnapshotError::Integrity */
/* Logical views (src/error.rs:65-77). */
#define B2F_ERR_LAYOUT_ZERO_STRIDE 22            /* FftError::BufferLayoutZeroStride */
#define B2F_ERR_LAYOUT_BATCH_STRIDE_TOO_SMALL 23 /* FftError::BufferLayoutBatchStrideTooSmall */
#define B2F_ERR_LAYOUT_OUT_OF_BOUNDS 24          /* FftError::BufferLayoutOutOfBounds */
#define B2F_ERR_LAYOUT_TOO_LARGE 25              /* FftError::BufferLayoutTooLarge */

/* FftDirection (src/config.rs:43-57). */
#define B2F_FORWARD 0
#define B2F_INVERSE 1
/* Normalization (src/config.rs:61-71); the crate's default is INVERSE. */
#define B2F_NORM_NONE 0
#define B2F_NORM_FORWARD 1
#define B2F_NORM_INVERSE 2
#define B2F_NORM_ORTHOGONAL 3
/* FftPrecision (src/config.rs:6-38). */
#define B2F_F32 0
#define B2F_F64 1
#define B2F_DF64 2
/* FftTransformKind. */
#define B2F_C2C 0
#define B2F_R2C 1
#define B2F_C2R 2

typedef struct b2f_config b2f_config;
typedef struct b2f_plan b2f_plan;
typedef struct b2f_recorder b2f_recorder;

/* ------------------------------------------------------------ FftConfig */

/* FftConfig::new_nd (src/config.rs:90-103): every axis, batch 1, forward,
 * Normalization::Inverse, f32, default tuning. */
b2f_status b2f_config_new(b2f_config** out, const uint64_t* shape, uint32_t rank);
void b2f_config_free(b2f_config* cfg);
/* FftConfig::with_axes (src/config.rs:122). */
b2f_status b2f_config_set_axes(b2f_config* cfg, const uint32_t* axes, uint32_t count);
/* FftConfig::with_batch (src/config.rs:127). */
b2f_status b2f_config_set_batch(b2f_config* cfg, uint64_t batch);
/* FftConfig::with_direction (src/config.rs:112). */
b2f_status b2f_config_set_direction(b2f_config* cfg, int32_t direction);
/* FftConfig::with_normalization (src/config.rs:117). */
b2f_status b2f_config_set_normalization(b2f_config* cfg, int32_t normalization);
/* FftConfig::with_precision (src/config.rs:132). */
b2f_status b2f_config_set_precision(b2f_config* cfg, int32_t precision);
/* FftTuning::with_<key> (src/tuning.rs:177-268) for the scalar knobs:
 * workgroup_size, fused_workgroup_size, rader_max_prime, direct_max_prime,
 * fused_min_convolution_length, fuse_long_axes, fuse_small_volumes,
 * large_chunk_max_batches, grouped_batch, swap_to_2_stage_4_step,
 * swap_to_3_stage_4_step, segmented_burst_depth,
 * max_storage_buffer_binding_size, max_buffer_size (0 = None for the
 * optional ones), large_route (0 auto, 1 force-chunk, 2 force-four-step,
 * 3 force-segmented); and the B200 knobs lines_per_block (0 = planner's
 * choice), threads_per_block (0 = planner's choice), twiddle_table (1 =
 * stage twiddles from an FP64-built table, 0 = computed in-kernel),
 * tensor_cores (1 = length-64 f32 lines on the tcgen05 layer) and
 * radix_order (stage order of the shared-memory engine: 0 = the planner's,
 * radix 16 first; 1 = reversed; nonzero keeps a line off the register
 * kernel) and tma_tiles (1 = f32 column-tile passes of <= 256 points staged
 * through the Tensor Memory Accelerator in a persistent grid; 0, the
 * default = plain loads, measured faster: these passes are bound by
 * instruction issue, not by load latency). */
b2f_status b2f_config_set_tuning(b2f_config* cfg, const char* key, int64_t value);
/* FftTuning::with_force_rader_axes / with_force_bluestein_axes
 * (src/tuning.rs:197-205): key "force_rader_axes" or "force_bluestein_axes". */
/* Reads back one scalar FftTuning field (same keys as b2f_config_set_tuning). */
b2f_status b2f_config_get_tuning(const b2f_config* cfg, const char* key, int64_t* value);
b2f_status b2f_config_set_tuning_axes(b2f_config* cfg, const char* key, const uint32_t* axes,
                                      uint32_t count);
/* FftConfig::validate (src/config.rs:178-211). */
b2f_status b2f_config_validate(const b2f_config* cfg);
/* FftConfig::required_buffer_size_bytes (src/config.rs:255-260). */
b2f_status b2f_config_required_buffer_size_bytes(const b2f_config* cfg, uint64_t* out);
/* FftConfig::scale / scale_f64 (src/config.rs:262-286). */
b2f_status b2f_config_scale(const b2f_config* cfg, float* out_f32, double* out_f64);

/* -------------------------------------------------------------- FftPlan */

/* FftPlan::c2c / r2c / c2r (src/plan.rs:221, 327, 355).  The plan binds to
 * CUDA device `device` (-1 = the calling thread's current device), builds
 * its tables and workspace there and keeps them until b2f_plan_free. */
b2f_status b2f_plan_c2c(b2f_plan** out, const b2f_config* cfg, int32_t device);
b2f_status b2f_plan_r2c(b2f_plan** out, const b2f_config* cfg, int32_t device);
b2f_status b2f_plan_c2r(b2f_plan** out, const b2f_config* cfg, int32_t device);
void b2f_plan_free(b2f_plan* plan);

/* FftPlan::kind (src/plan.rs:390): B2F_C2C, B2F_R2C or B2F_C2R. */
int32_t b2f_plan_kind(const b2f_plan* plan);
/* FftPlan::required_buffer_size_bytes and the input/output forms
 * (src/plan.rs:462-484). */
uint64_t b2f_plan_required_buffer_size_bytes(const b2f_plan* plan);
uint64_t b2f_plan_required_input_buffer_size_bytes(const b2f_plan* plan);
uint64_t b2f_plan_required_output_buffer_size_bytes(const b2f_plan* plan);
/* FftPlan::workspace_size_bytes (src/plan.rs:446): device memory the plan
 * holds for multi-pass routes (allocated by the plan). */
uint64_t b2f_plan_workspace_size_bytes(const b2f_plan* plan);
/* FftPlan::supports_in_place (src/plan.rs:815). */
int32_t b2f_plan_supports_in_place(const b2f_plan* plan);

/* FftPlan::execute_checked (src/plan.rs:510-518): transform `in` into `out`
 * on `stream`.  The input buffer is left unchanged. */
b2f_status b2f_plan_execute_checked(const b2f_plan* plan, void* stream, const void* in,
                                    uint64_t in_bytes, void* out, uint64_t out_bytes);
/* FftPlan::execute_in_place (src/plan.rs:827-835). */
b2f_status b2f_plan_execute_in_place(const b2f_plan* plan, void* stream, void* buffer,
                                     uint64_t bytes);
/* FftPlan::diagnostics (src/plan.rs:938-1003) as JSON: route, axis kinds,
 * factors, stages (label, kind, route, radix schedule, launch shape),
 * buffer requirements and requested/effective tuning.  On entry *len is the
 * capacity of buf; on return it is the length needed (without the NUL). */
b2f_status b2f_plan_diagnostics_json(const b2f_plan* plan, char* buf, uint64_t* len);
/* No counterpart in the crate (wgpu reports device loss through its own
 * callbacks): waits for the plan's device work (synchronising its device)
 * and reports whether a bounded device-side wait of its kernels gave up
 * (the tensor-core layer's waits for its matrix products), clearing the
 * flag.  B2F_OK when none did, else B2F_ERR_DEVICE with the detail. */
b2f_status b2f_plan_device_status(const b2f_plan* plan);

/* FftLogicalLayout (src/runtime/logical_io.rs:34-38, 90-110): logical
 * element i of batch b sits at element element_offset + b * batch_stride +
 * i * element_stride of the buffer, counted in the endpoint's elements (a
 * complex value of the plan's precision; a real value on the real side of
 * an R2C/C2R plan).  element_stride 0 is rejected (BufferLayoutZeroStride);
 * batch_stride 0 means None, i.e. the per-batch span
 * element_stride * (elements - 1) + 1, and a smaller nonzero value is
 * rejected (BufferLayoutBatchStrideTooSmall). */
typedef struct b2f_logical_layout {
  uint64_t element_offset;
  uint64_t element_stride;
  uint64_t batch_stride;
} b2f_logical_layout;

/* FftPlan::execute_logical_views / execute_views (src/plan.rs:580-806):
 * the plan between two caller views.  A NULL layout is the contiguous view
 * (offset 0, stride 1).  A wgpu BufferView (buffer, offset, size) is the
 * pointer advanced by the offset with its size: execute_views needs no
 * separate entry point.  Contiguous and offset-only layouts run on the
 * caller's memory directly; strided layouts gather the input into, and/or
 * scatter the output from, staging buffers the plan allocates on first use
 * and keeps.  Sizes: the view must hold offset + (batch - 1) * batch_stride
 * + span elements (BufferLayoutOutOfBounds otherwise). */
b2f_status b2f_plan_execute_logical_views(const b2f_plan* plan, void* stream, const void* in,
                                          uint64_t in_bytes, const b2f_logical_layout* in_layout,
                                          void* out, uint64_t out_bytes,
                                          const b2f_logical_layout* out_layout);

/* ---------------------------------------------------------- FftRecorder */

/* FftRecorder::new (src/plan.rs:72-83): starts capturing the work of the
 * following record calls on `stream` into one CUDA graph, the B200
 * counterpart of the crate's shared compute pass. */
b2f_status b2f_recorder_begin(b2f_recorder** out, void* stream);
/* FftPlan::record (src/plan.rs:882-895). */
b2f_status b2f_plan_record(const b2f_plan* plan, b2f_recorder* rec, const void* in,
                           uint64_t in_bytes, void* out, uint64_t out_bytes);
/* FftPlan::record_in_place (src/plan.rs:839-879). */
b2f_status b2f_plan_record_in_place(const b2f_plan* plan, b2f_recorder* rec, void* buffer,
                                    uint64_t bytes);
/* Ends the capture and instantiates the graph (the crate's encoder.finish). */
b2f_status b2f_recorder_finish(b2f_recorder* rec);
/* Launches the recorded graph on `stream` (the crate's queue.submit). */
b2f_status b2f_recorder_submit(b2f_recorder* rec, void* stream);
void b2f_recorder_free(b2f_recorder* rec);

/* ------------------------------------------------------- batched launch */

/* Many 1D complex f32 transforms of mixed lengths in one persistent launch
 * (no counterpart in the crate, which records one dispatch chain per plan):
 * line i has lengths[i] points at complex offset offsets[i] of the input and
 * output buffers (lines must not overlap); direction and normalization are
 * shared.  Lines that fit one CTA are taken from a device work queue by
 * persistent CTAs; longer lines run as a column pass and a row pass (three
 * passes for Bluestein lengths) through a scratch region, their column and
 * row groups taken from a second work queue. */
typedef struct b2f_batch b2f_batch;
b2f_status b2f_batch_new(b2f_batch** out, const uint64_t* lengths, const uint64_t* offsets,
                         uint64_t count, int32_t direction, int32_t normalization,
                         int32_t device);
/* b2f_batch_new with flags: bit 0 (B2F_BATCH_CLUSTERS) runs lines too long
 * for one CTA on 8/16-CTA thread-block clusters that keep the whole line in
 * distributed shared memory (one HBM pass, fewer lines in flight) instead
 * of the default column and row passes through a scratch region. */
#define B2F_BATCH_CLUSTERS 1u
b2f_status b2f_batch_new_ex(b2f_batch** out, const uint64_t* lengths, const uint64_t* offsets,
                            uint64_t count, int32_t direction, int32_t normalization,
                            int32_t device, uint32_t flags);
void b2f_batch_free(b2f_batch* batch);
/* Bytes each of the input and output buffers must hold. */
uint64_t b2f_batch_required_buffer_size_bytes(const b2f_batch* batch);
/* Transforms every line of `in` into `out` (in == out allowed). */
b2f_status b2f_batch_execute(const b2f_batch* batch, void* stream, const void* in,
                             uint64_t in_bytes, void* out, uint64_t out_bytes);
/* b2f_batch_execute restricted to a subset of the lines, for measuring one
 * kernel alone: parts bit 0 = lines that fit one CTA, bit 1 = cluster lines,
 * bit 2 = the column/row passes of the other long lines; sequential != 0
 * runs the cluster kernels on `stream` too instead of a second stream. */
b2f_status b2f_batch_execute_parts(const b2f_batch* batch, void* stream, const void* in,
                                   uint64_t in_bytes, void* out, uint64_t out_bytes,
                                   uint32_t parts, int32_t sequential);
/* b2f_batch_execute from and to host memory: the lines are cut, in offset
 * order, into chunks of about 32 MiB (at most 32; with 8 or more, the
 * first three and the last three hold 1/8, 1/4 and 1/2 of the others'
 * share, to shorten the pipeline's fill and drain), and chunk c's copy in
 * (host_in -> dev_in), transform (dev_in -> dev_out) and copy out
 * (dev_out -> host_out) overlap the other chunks' on three internal
 * streams; `stream` orders the whole call with the caller's work (the call
 * is asynchronous: the results are in host_out once `stream` has reached
 * this point).  Each of the four buffers holds `bytes` >=
 * b2f_batch_required_buffer_size_bytes; host_in == host_out and dev_in ==
 * dev_out are allowed.  Host buffers should be page-locked for the copies
 * to overlap.  The copies are cut at 4 KiB multiples of the buffers'
 * offsets, so unused bytes between lines within 4 KiB of a chunk boundary
 * are copied too (their values in host_out are unspecified).  Batches with cluster lines (B2F_BATCH_CLUSTERS) run
 * unchunked: copy in, execute, copy out. */
b2f_status b2f_batch_execute_host(const b2f_batch* batch, void* stream, const void* host_in,
                                  void* host_out, void* dev_in, void* dev_out, uint64_t bytes);
/* Task and launch summary as JSON (same length convention as the plan's). */
b2f_status b2f_batch_diagnostics_json(const b2f_batch* batch, char* buf, uint64_t* len);

/* -------------------------------------------------------------- serving */

/* Serving loop (no counterpart in the crate): a scheduler thread that keeps
 * plans, tables and workspaces resident, admits requests by an HBM budget,
 * and batches continuously (arrivals join the next group while earlier
 * ones run), overlapping groups on `nstreams` streams.  1D complex f32
 * requests of one direction and normalization are coalesced whatever their
 * lengths into one batched launch of the mixed-length line kernels; other
 * requests of the same configuration are coalesced into one execution of a
 * resident plan (plans keyed by configuration and a power-of-two batch
 * bucket, or by the exact batch once a batch recurs; evicted least recently
 * used when the budget needs the room).  A lone 1D request runs on a plan.
 * Plans are built on the scheduler thread with its lock released, so
 * submits and waits never stall behind a build; the group that needs the
 * plan waits for it.  Requests carry host buffers (pinned memory lets the copies overlap;
 * results are written back to host_out) or device buffers
 * (b2f_server_submit_device).  When a group fails, no copy touching a
 * request's memory is pending by the time its wait returns the error.
 * hbm_budget_bytes 0 = 120 GB.  The server raises the release threshold of
 * the device's default memory pool to its budget (never lowers it), so the
 * groups' stream-ordered allocations stay mapped across synchronisations. */
typedef struct b2f_server b2f_server;
b2f_status b2f_server_new(b2f_server** out, int32_t device, uint64_t hbm_budget_bytes,
                          int32_t nstreams, int32_t coalesce);
void b2f_server_free(b2f_server* server);
/* Queues one transform (kind B2F_C2C / B2F_R2C / B2F_C2R of `cfg`). */
b2f_status b2f_server_submit(b2f_server* server, const b2f_config* cfg, int32_t kind,
                             const void* host_in, uint64_t in_bytes, void* host_out,
                             uint64_t out_bytes, uint64_t* request_id);
/* b2f_server_submit with the request's buffers in device memory of the
 * server's device: the transform reads and writes them where they lie (no
 * host copies).  1D complex f32 requests need 8-byte aligned buffers to
 * join a batched line launch; others run alone. */
b2f_status b2f_server_submit_device(b2f_server* server, const b2f_config* cfg, int32_t kind,
                                    const void* dev_in, uint64_t in_bytes, void* dev_out,
                                    uint64_t out_bytes, uint64_t* request_id);
/* Blocks until the request completed (or timeout_s passed; 0 = 1 hour). */
b2f_status b2f_server_wait(b2f_server* server, uint64_t request_id, double timeout_s);
/* Blocks until nothing is queued or in flight (while dispatch is held,
 * until it is released or timeout_s passes). */
b2f_status b2f_server_drain(b2f_server* server, double timeout_s);
/* hold != 0: requests are queued but not dispatched; hold == 0 releases
 * them, coalesced, so a burst submitted between the two forms as few
 * groups as its keys allow.  Closing the server dispatches what is queued. */
void b2f_server_hold(b2f_server* server, int32_t hold);
/* Completed/failed counts, groups, coalesced requests, p50/p99 latency
 * (submission to completion), requests/s and FFTs/s over the served span,
 * HBM in use, resident plans; same length convention as the plan's. */
b2f_status b2f_server_stats_json(b2f_server* server, char* buf, uint64_t* len);
void b2f_server_reset_stats(b2f_server* server);

/* ---------------------------------------------------- allocation-free */

/* No counterpart in the crate.  For callers that cannot allocate device
 * memory -- code recording a CUDA graph whose capture forbids allocation, a
 * plug-in running inside a host application that owns a fixed device-memory
 * budget, a real-time path that must not take the allocator's locks or wait
 * on its synchronisation -- this transforms `batch` 1D complex f32 lines of
 * n points (n 2,3,5,7,11,13-smooth) from `in` to `out` without any
 * allocation: no plan object, no tables (stage twiddles are computed in the
 * kernels), and lines too long for one CTA run their two four-step passes
 * through a static device array of 32 MiB inside the library.  Limit: the
 * multi-pass route takes n * batch <= 4,194,304 points (32 MiB of f32
 * complex); above it the call returns B2F_ERR_WORKSPACE_TOO_SMALL.  Every
 * GPU that loads the library holds the 32 MiB array until the process
 * exits.  The first call on each device looks the array's device address
 * up (cudaGetSymbolAddress, with that device current); make that first
 * call before any stream capture.  The address is cached for the life of
 * the device's primary context: calling cudaDeviceReset on a device
 * invalidates it, so this entry point must not be used after one.  All calls share the one array (the last
 * call's contents stay in it; every element is rewritten before it is read,
 * so nothing needs clearing), so calls that overlap on the GPU race: issue
 * them on one stream, or order them.  Inputs, outputs, direction and
 * normalization are the caller's, as in b2f_plan_execute_checked. */
b2f_status b2f_c2c_1d_f32_noalloc(void* stream, const void* in, uint64_t in_bytes, void* out,
                                  uint64_t out_bytes, uint64_t n, uint64_t batch,
                                  int32_t direction, int32_t normalization);

/* ---------------------------------------------------------- df64 canary */

/* validate_df64_invariants (src/df64_canary.rs:1-8, 101-235): evaluates the
 * df64 route's error-free transforms (two-sum, quick-two-sum, two-product,
 * df64 add and multiply, complex add and multiply, an overflow-edge
 * product, a constant product) on the device on 4 adversarial input cases
 * and compares each of the 88 f32 words bit for bit with the same
 * transforms in IEEE single precision on the host.  Returns B2F_OK when all
 * match; otherwise B2F_ERR_DEVICE with "InvariantMismatch { case, word,
 * actual, expected }" in b2f_last_error_message.  words (nullable) receives
 * the 88 device words; *exact_words (nullable) the count that matched
 * before the first mismatch.  device -1 = the current device. */
b2f_status b2f_df64_canary(int32_t device, uint32_t* words, uint64_t* exact_words);

/* --------------------------------------------------------------- errors */

/* FftError's Display (src/error.rs): a fixed name for each status. */
/* ------------------------------------------- autotuner and tuning snapshot */

/* Autotuner (the batching form's "autotuner + tuning snapshot"; nearest
 * reference ancestors: FftTuning, src/tuning.rs:35-268, and the pipeline
 * cache snapshot, src/runtime/pipeline_cache.rs:14-395).  Creates the plan of
 * `cfg` (kind B2F_C2C/R2C/C2R) on `device`, times it and candidate tunings
 * of the kernel-shape knobs (twiddle_table, then radix_order, then
 * lines_per_block 1..16, then threads_per_block 64..512; `reps` executions each after two warm-ups, 0 =
 * 20) on buffers it allocates and fills with deterministic values, keeps the
 * fastest candidate whose output matches the default plan's within the
 * precision's tolerance (f32 2e-6, f64 1e-13, df64 1e-12 relative L2), and
 * records it in the process-wide tuning snapshot.  The report (JSON: key,
 * default_us, best_us, best, every candidate with its time and error) is
 * written to report as b2f_plan_diagnostics_json does. */
b2f_status b2f_autotune(const b2f_config* cfg, int32_t kind, int32_t device, uint32_t reps,
                        char* report, uint64_t* len);
/* Records a tuning for cfg's key by hand (validated like a plan's tuning). */
b2f_status b2f_tuning_snapshot_record(const b2f_config* cfg, int32_t kind, int64_t lines_per_block,
                                      int64_t threads_per_block, int64_t twiddle_table,
                                      int64_t radix_order, double best_us, double default_us);
/* Copies the snapshot's tuning for cfg's key into cfg; *found = 0 or 1. */
b2f_status b2f_tuning_snapshot_apply(b2f_config* cfg, int32_t kind, int32_t* found);
/* The snapshot as versioned JSON (schema "wgpufft_b200.tuning", version 2,
 * device, entries ordered by key, FNV-1a checksum over device and entries). */
b2f_status b2f_tuning_snapshot_json(char* buf, uint64_t* len);
b2f_status b2f_tuning_snapshot_save(const char* path);
/* Replaces the snapshot with the file's after checking it: JSON syntax and
 * fields (SnapshotJson), schema (SnapshotSchemaMismatch), version
 * (SnapshotVersionMismatch), and integrity (SnapshotIntegrity): every key
 * canonical and re-derived from its fields, keys strictly ordered (no
 * duplicates), tuning values valid for their configuration, checksum, and,
 * with device >= 0, entries measured on a device of the same name and
 * architecture.  On any error the snapshot in memory is unchanged. */
b2f_status b2f_tuning_snapshot_load(const char* path, int32_t device);
void b2f_tuning_snapshot_clear(void);

const char* b2f_status_string(b2f_status status);
/* Detail of the calling thread's last failure; returns its length and
 * copies at most len-1 bytes plus a NUL into buf (buf may be NULL). */
uint64_t b2f_last_error_message(char* buf, uint64_t len);
/* Library version string. */
const char* b2f_version(void);

#ifdef __cplusplus
}
#endif

#endif /* WGPUFFT_B200_H */
