/*
 * tilestream_c.h - the C entry points of libtilestream_b200.so.
 *
 * A flat C ABI over the drop-in C++ API of include/tilestream/ (plain pointers, sizes and POD
 * records; no C++ or torch types). Every record below has exactly the layout of the C++ record
 * it mirrors (checked with static_asserts in the library), and every function returns the
 * reference's Status value (include/tilestream/types.h: 0 = success ... 10 = io_error).
 * Streams are CUDA stream handles (cudaStream_t) passed as void*.
 *
 * Each declaration names the reference interface it replaces (path:line in the reference).
 */
#ifndef TILESTREAM_C_H
#define TILESTREAM_C_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- records (include/tilestream/types.h:21-71, cuda.h:16-109) ------------------------- */
typedef struct { uint32_t type, width, height; } ts_image_spec;    /* ImageSpec */
typedef struct { uint16_t width, height; } ts_tile_shape;         /* TileShape */
typedef struct { uint32_t x, y, width, height; } ts_roi;          /* Roi */
typedef struct { const void *data; uint64_t size; } ts_const_bytes;
typedef struct { void *data; uint64_t size; } ts_mutable_bytes;
typedef struct {
    const void *data;
    ts_image_spec image;
    uint64_t pitch_bytes, capacity_bytes;
} ts_const_image_view;
typedef struct {
    void *data;
    ts_image_spec image;
    uint64_t pitch_bytes, capacity_bytes;
} ts_image_view;
typedef struct { uint32_t status, reserved; uint64_t bytes_written; } ts_device_result;
typedef struct { uint32_t kind; float scalar; ts_const_image_view map; } ts_parameter;
typedef struct { ts_parameter offset, gain; } ts_calibration;
typedef struct { uint64_t tile_index, input_offset; } ts_tile_mapping;
typedef struct { uint64_t file_bytes, tile_count, metadata_bytes; } ts_parse_limits;
typedef struct {
    uint64_t image_count, tile_count;
    ts_tile_shape tile;
    uint64_t scan_temp_bytes;
} ts_workspace_spec;
/* Host metadata tables (api.h:11-35): TileMetadata is 32 bytes, SegmentMetadata 24 bytes. */
typedef struct {
    uint32_t mode;
    uint16_t width, height;
    uint64_t offset, length, first_segment;
} ts_tile_metadata;
typedef struct {
    uint32_t seed, bit_width;
    uint64_t payload_offset, payload_bytes;
} ts_segment_metadata;

/* An owned tilestream::ImageMetadata (api.h:29-35). */
typedef struct ts_metadata ts_metadata;
/* An owned tilestream::cuda::BatchPlan (cuda.h:148-174). */
typedef struct ts_plan ts_plan;

typedef struct {
    ts_const_bytes bytes;
    const ts_metadata *metadata;
    const ts_tile_mapping *mappings;
    uint64_t mapping_count;
    const ts_device_result *encoder_result;
    ts_image_spec trusted_image;
    ts_tile_shape trusted_tile;
} ts_compressed_input; /* CompressedInput, cuda.h:42-51 */
typedef struct {
    ts_const_image_view input;
    ts_image_view output;
    ts_mutable_bytes compressed_output;
    ts_compressed_input compressed_input;
    ts_roi roi;
    ts_calibration calibration;
} ts_batch_item; /* BatchItem, cuda.h:53-60 */
typedef struct {
    uint32_t operation; /* 0 compress, 1 decompress, 2 decode_roi, 3 calibrate, 4 decode_calibrate */
    const ts_batch_item *items;
    uint64_t count;
    ts_tile_shape tile;
} ts_batch_request; /* BatchRequest, cuda.h:62-67 */
typedef struct { ts_device_result *data; uint64_t count; } ts_result_buffer; /* cuda.h:106-109 */

/* ---- size queries (sizing.h:26-30) ------------------------------------------------------ */
int ts_image_span(ts_image_spec image, uint64_t pitch_bytes, uint64_t *bytes);
int ts_compress_bound(ts_image_spec image, ts_tile_shape tile, uint64_t *bytes);
int ts_workspace_size(const ts_workspace_spec *spec, uint64_t *bytes);

/* ---- host parser (api.h:42-43) ------------------------------------------------------------
 * On success *out receives a new handle (free with ts_metadata_destroy); on failure *out is
 * left unchanged. limits may be NULL for no budget. */
int ts_parse_metadata(ts_const_bytes source, const ts_parse_limits *limits, ts_metadata **out);
/* Wraps caller-built tables (copied) as metadata for a GPU plan. */
int ts_metadata_create(ts_image_spec image, ts_tile_shape tile, uint64_t file_bytes,
                       const ts_tile_metadata *tiles, uint64_t tile_count,
                       const ts_segment_metadata *segments, uint64_t segment_count,
                       ts_metadata **out);
void ts_metadata_destroy(ts_metadata *metadata);
void ts_metadata_info(const ts_metadata *metadata, ts_image_spec *image, ts_tile_shape *tile,
                      uint64_t *file_bytes, uint64_t *tile_count, uint64_t *segment_count);
const ts_tile_metadata *ts_metadata_tiles(const ts_metadata *metadata);
const ts_segment_metadata *ts_metadata_segments(const ts_metadata *metadata);

/* ---- CPU codec (cpu.h:9-12) ---------------------------------------------------------------- */
int ts_cpu_compress(ts_const_image_view input, ts_tile_shape tile, ts_mutable_bytes output,
                    uint64_t *bytes_written);
int ts_cpu_decompress(ts_const_bytes input, ts_image_view output, const ts_parse_limits *limits);

/* ---- CUDA plans and executors (cuda.h:176-187) ---------------------------------------------
 * ts_prepare_batch replaces *plan (destroying the previous plan) only on success. */
int ts_prepare_batch(const ts_batch_request *request, ts_plan **plan, void *stream);
void ts_plan_destroy(ts_plan *plan);
int ts_plan_workspace_spec(const ts_plan *plan, ts_workspace_spec *spec); /* cuda.h:156 */
int ts_compress_async(const ts_plan *plan, ts_mutable_bytes workspace, ts_result_buffer results,
                      void *stream);
int ts_decompress_async(const ts_plan *plan, ts_mutable_bytes workspace, ts_result_buffer results,
                        void *stream);
int ts_decode_roi_async(const ts_plan *plan, ts_mutable_bytes workspace, ts_result_buffer results,
                        void *stream);
int ts_calibrate_async(const ts_plan *plan, ts_mutable_bytes workspace, ts_result_buffer results,
                       void *stream);
int ts_decode_calibrate_async(const ts_plan *plan, ts_mutable_bytes workspace,
                              ts_result_buffer results, void *stream);

/* ---- mixed batches (include/tilestream/batch.h; extension, no reference counterpart) -------
 * Many archives and ROIs with mixed pixel types, tile geometries and decode operations in one
 * persistent kernel over one device task queue, replayed as a CUDA graph, optionally tuned. */
typedef struct {
    uint32_t operation; /* 1 decompress, 2 decode_roi, 4 decode_calibrate */
    ts_batch_item item;
} ts_mixed_item; /* MixedItem */
typedef struct {
    uint32_t graph;         /* nonzero: executions replay a CUDA graph */
    uint32_t autotune;      /* nonzero: time candidate kernel shapes and grids at preparation */
    const char *tune_cache; /* file remembering tuned choices, or NULL */
    int32_t shape;          /* a fixed kernel shape, 0 .. ts_decode_shape_count() - 1; -1: default */
} ts_mixed_options;
uint32_t ts_decode_shape_count(void);
typedef struct {
    uint64_t tiles;
    uint32_t shape, grid, per_sm, graph;
    float tuned_us;
} ts_mixed_stats;
typedef struct ts_mixed_batch ts_mixed_batch;

/* Results: one record per item, bound at preparation. *batch is replaced only on success. */
int ts_prepare_mixed_batch(const ts_mixed_item *items, uint64_t count, ts_result_buffer results,
                           const ts_mixed_options *options, ts_mixed_batch **batch, void *stream);
int ts_run_mixed_batch(const ts_mixed_batch *batch, void *stream);
int ts_mixed_batch_stats(const ts_mixed_batch *batch, ts_mixed_stats *stats);
void ts_mixed_batch_destroy(ts_mixed_batch *batch);

/* ---- ROI serving (include/tilestream/serve.h; extension, no reference counterpart) ---------
 * Resident archives, requests admitted by output-pool memory and batched into one persistent
 * decoder launch each, several launches in flight. Archive bytes and metadata must outlive the
 * server. */
typedef struct {
    uint32_t archive;
    ts_roi roi;
    uint32_t calibrated; /* nonzero: FP32 output RN(RN(x - offset) * gain) */
    float offset, gain;
    double arrival_us; /* after the start of the run; non-decreasing */
} ts_serve_request; /* ServeRequest */
typedef struct {
    uint64_t output_pool_bytes;
    uint32_t max_batch;    /* requests per launch, 1-48 */
    uint32_t max_inflight; /* launches on the GPU at once, 1-16 */
    uint64_t max_batch_tiles;
    uint32_t retain_outputs; /* nonzero: outputs stay valid until the run ends */
    uint32_t serial;         /* nonzero: one request at a time through the plan API */
} ts_serve_options; /* ServeOptions */
typedef struct {
    double wall_us, throughput_rps, decoded_gbs;
    double p50_us, p90_us, p99_us, max_us, mean_us;
    uint64_t completed, rejected, batches;
    double mean_batch;
    uint64_t max_inflight, stalls, tiles, output_bytes;
} ts_serve_stats; /* ServeStats */
typedef struct {
    double latency_us, queued_us;
    uint64_t output_offset, output_pitch;
    uint32_t batch_size;
    ts_device_result result;
} ts_serve_outcome; /* ServeOutcome */
typedef struct ts_server ts_server;

/* options NULL: defaults. *server is replaced only on success. */
int ts_server_create(const ts_serve_options *options, ts_server **server);
int ts_server_add_archive(ts_server *server, ts_const_bytes device_bytes,
                          const ts_metadata *metadata, uint32_t *id);
int ts_server_seal(ts_server *server);
int ts_server_run(ts_server *server, const ts_serve_request *requests, uint64_t count,
                  ts_serve_outcome *outcomes, ts_serve_stats *stats);
int ts_server_pool(const ts_server *server, ts_mutable_bytes *pool);
/* Sessions (Server::start/submit/wait/release/stop): requests submitted from any thread while
 * the serving loop runs on a thread of its own. submit, wait and release are thread-safe; wait
 * returns 0 with *done = 0 when timeout_us passes first. */
int ts_server_start(ts_server *server, uint32_t max_outstanding);
int ts_server_submit(ts_server *server, const ts_serve_request *request, uint64_t *ticket);
int ts_server_wait(ts_server *server, uint64_t ticket, uint64_t timeout_us,
                   ts_serve_outcome *outcome, int *done);
int ts_server_release(ts_server *server, uint64_t ticket);
int ts_server_stop(ts_server *server);
void ts_server_destroy(ts_server *server);

/* ---- ROI staging from an archive outside the GPU (include/tilestream/staging.h) ------------
 * No counterpart in the reference API (its benchmark gathers an ROI's tiles with host copies,
 * benchmarks/codec_benchmark.cpp:153-320). ts_stage_roi_tiles enqueues on stream the copies of
 * the payloads of the tiles that intersect roi, from archive (the whole .tsc file, pinned host
 * or device memory) into staging (device memory), one run of adjacent payloads per tile row of
 * a parsed file (one small kernel for all of them when the archive is pinned or on the device,
 * one copy per run when it is pageable), and writes one ts_tile_mapping per tile for a
 * decode_roi or decode_calibrate item on a stream ordered after the copies. */
typedef struct { uint64_t tiles, bytes, copies; } ts_roi_staging; /* RoiStaging */
int ts_roi_staging_size(const ts_metadata *metadata, ts_roi roi, ts_roi_staging *out);
int ts_stage_roi_tiles(const ts_metadata *metadata, ts_roi roi, ts_const_bytes archive,
                       ts_mutable_bytes staging, ts_tile_mapping *mappings,
                       uint64_t mapping_capacity, void *stream, ts_roi_staging *out);

/* ---- allocation-free encode (no counterpart in the reference) ------------------------------
 * Encodes one image into a complete .tsc file on the GPU, like a one-item compress plan, but
 * allocates no memory: no plan tables, no workspace, no cudaMalloc or cudaFree. It is for
 * callers that cannot allocate device memory while they encode - a process whose GPU memory is
 * fully reserved by another allocator, an acquisition loop that must not stall on an allocator
 * or an implicit device synchronization, a deployment that forbids dynamic allocation after
 * initialization. Its scratch is a fixed 1056 KiB array in device memory that the library holds
 * on every GPU it is loaded on, which limits one image to ts_compress_noalloc_max_tiles()
 * tiles (131,070: for example 16384 x 32768 pixels with 128x32 tiles); larger images return
 * resource_limit and nothing is written.
 *
 * input, output and result are device memory of the current device; output needs
 * compress_bound bytes and result one ts_device_result. Arguments are checked as for
 * compress_async, statuses are the same, and per-image completion is written to *result.
 * The first call on each device loads the kernels there and sizes their grid, and must
 * therefore come before any stream capture on that device; every call looks up the device's
 * address of the array afresh. Every call shares the array and clears what it uses:
 * calls that overlap on one GPU race, so order them on one stream or with events. */
int ts_compress_noalloc(ts_const_image_view input, ts_tile_shape tile, ts_mutable_bytes output,
                        ts_device_result *result, void *stream);
uint64_t ts_compress_noalloc_max_tiles(void);

/* ---- unparsed files (include/tilestream/unparsed.h; extension, no reference counterpart) ---
 * Whole-image decode of .tsc files in device memory that were never parsed on the host: the
 * host checks each header from its 64-byte host copy, the decoder validates index entries,
 * payloads and rows on the device with parse_metadata's rules. At most 16 files per call. */
typedef struct {
    ts_const_bytes bytes; /* device memory: the whole file */
    const void *header;   /* host copy of its first 64 bytes */
    ts_image_view output; /* device memory */
} ts_unparsed_file;       /* UnparsedFile */
int ts_decode_unparsed_async(const ts_unparsed_file *files, uint64_t count,
                             ts_result_buffer results, void *stream);

/* ---- TIFF import and export (include/tilestream/tiff.h; reference tiff.h:10-37) --------- */
typedef struct {
    uint32_t max_width, max_height;
    uint64_t max_decoded_bytes;
} ts_tiff_read_limits; /* TiffReadLimits */
typedef struct {
    uint32_t bigtiff;              /* nonzero: BigTIFF */
    uint32_t compression;          /* 0 none, 1 deflate */
    uint32_t horizontal_predictor; /* nonzero: predictor 2 (uint16 + deflate only) */
    uint32_t tile_width, tile_height, deflate_level;
} ts_tiff_write_options; /* TiffWriteOptions, field by field */
/* An owned tilestream::io::TiffImage. */
typedef struct ts_tiff_image ts_tiff_image;

/* io::read_tiff (tiff.h:34-35). limits NULL: none. *image is replaced only on success. */
int ts_read_tiff(const char *path, const ts_tiff_read_limits *limits, ts_tiff_image **image);
/* The image's spec, row pitch and packed pixels (host memory owned by the image). */
int ts_tiff_image_pixels(const ts_tiff_image *image, ts_image_spec *spec, uint64_t *pitch_bytes,
                         const void **pixels, uint64_t *bytes);
void ts_tiff_image_destroy(ts_tiff_image *image);
/* io::write_tiff (tiff.h:36-37); image is host memory. options NULL: defaults. */
int ts_write_tiff(const char *path, ts_const_image_view image,
                  const ts_tiff_write_options *options);

/* ---- plan inspection (extension, no reference counterpart) ---------------------------------
 * For validation tooling. Runs the host half of ts_prepare_batch for a decode request
 * (decompress, decode_roi or decode_calibrate): every argument, metadata, ROI, capacity and
 * aliasing check that needs no device, then the planning of its tile tasks. It never touches
 * a device and dereferences no buffer pointer, so any address values may stand in for device
 * buffers. Returns the status of those checks (device and pointer checks are not made).
 * *count receives the number of tasks; the first min(*count, capacity) are described:
 *   read_begin/read_end    the bytes the task stages (a parsed tile's payload; for an
 *                          encoder-output source, the whole archive buffer, whose index entry
 *                          and row descriptors the kernel validates itself)
 *   write_begin/write_end  the first and one past the last output byte it may write
 *   rows_end               parsed predictive tiles: one past the furthest row descriptor,
 *                          relative to read_begin (0 otherwise)
 *   mode, flags            the tile mode (0 raw, 1 constant, 2 predict) and task flags
 *                          (1 FP32, 2 calibrated, 4 encoder output, 8 first of its image,
 *                          16 whole aligned rows) */
typedef struct {
    uint64_t image;
    uint64_t read_begin, read_end;
    uint64_t write_begin, write_end;
    uint64_t rows_end;
    uint32_t mode, flags;
    uint32_t width, height;
} ts_task_span;
int ts_inspect_decode(const ts_batch_request *request, ts_task_span *spans, uint64_t capacity,
                      uint64_t *count);

/* ---- device buffers and completion (cuda.h:113-145) ----------------------------------------
 * Stream-ordered allocation aligned to 256 bytes; *data is replaced only on success. */
int ts_device_allocate(uint64_t bytes, void *stream, void **data);
int ts_device_release(void *data, void *stream);
int ts_synchronize(void *stream);

/* ---- library information (info.h:7-8) ----------------------------------------------------- */
const char *ts_version(void);
/* Copies the JSON report (NUL-terminated) into buf when it fits; *needed gets its size + 1. */
int ts_info_json(char *buf, uint64_t capacity, uint64_t *needed);

#ifdef __cplusplus
}
#endif

#endif /* TILESTREAM_C_H */
