// Execution records shared by the host planner and the sm_100a kernels, and the internal
// extern "C" launcher layer between them. Plain C layout: no C++ types cross this boundary.
//
// The planner flattens every batch into one queue of self-contained tile tasks, so a kernel
// never searches for the image that owns a block (the reference binary-searches window entries
// per block, src/cuda/device.cuh:32-45).
#pragma once

#include <cuda_runtime_api.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    TSK_RAW = 0,
    TSK_CONSTANT = 1,
    TSK_PREDICT = 2,
};

// DecodeTask.flags
enum {
    TSK_F32 = 1,        // samples are FP32 words (else uint16)
    TSK_CALIBRATED = 2, // output is calibrated FP32
    TSK_TRUSTED = 4,    // index entry and rows are read on the device (encoder output)
    TSK_FIRST = 8,      // first task of its image: writes the image's result record
    TSK_FULL = 16,      // every column of full-width rows is written, to 16-byte-aligned rows
    TSK_UNPARSED = 32,  // with TSK_TRUSTED: a file never parsed on the host, validated on the
                        // device with the host parser's rules (no producing result record)
};

// Largest payload of one tile: RAW FP32, 4096 samples.
#define TSK_TILE_PIXELS 4096
#define TSK_MAX_ROWS 64
#define TSK_PAYLOAD_BYTES 16384

// One tile to decode. 64 bytes, self-contained: a consumer needs nothing else but the payload.
typedef struct __align__(16) {
    // Parsed: device address of the tile payload. Trusted: device address of the archive.
    uint64_t src;
    // Parsed: payload length in 32-bit words. Trusted: the tile's index in the archive.
    uint64_t words_or_tile;
    // Output address of tile column 0 in tile row row0 (may lie before the region when the ROI
    // starts inside the tile; only columns [col0, col1) are written), and the output pitch.
    uint64_t dst;
    uint64_t pitch;
    uint32_t image;   // slot in the image table and the result buffer
    uint32_t rows_at; // parsed PREDICT: first entry of this tile's row table
    uint32_t ox;      // output column of tile column col0 (calibration maps)
    uint32_t oy;      // output row of tile row row0 (calibration maps)
    uint16_t width;   // actual tile width
    uint16_t height;  // actual tile height
    uint16_t row0, row1; // tile rows written: [row0, row1)
    uint16_t col0, col1; // tile columns written: [col0, col1)
    uint8_t mode;        // parsed: TSK_RAW/CONSTANT/PREDICT
    uint8_t flags;
    uint16_t reserved;
} tsk_decode_task;

// Per-image state of a decode execution. 96 bytes.
typedef struct __align__(16) {
    uint64_t out;   // output base (device address)
    uint64_t out_pitch;
    uint64_t offset_map; // 0 when the offset is a scalar
    uint64_t offset_pitch;
    uint64_t gain_map; // 0 when the gain is a scalar
    uint64_t gain_pitch;
    uint64_t result_bytes;   // bytes_written reported on success
    uint64_t encoder_result; // trusted: producing DeviceResult (device address), else 0
    uint64_t capacity;       // trusted: capacity of the archive buffer in bytes
    float offset;
    float gain;
    uint32_t tile_count; // tasks of this image (trusted completion count)
    uint32_t archive_width;  // trusted: archive geometry
    uint32_t archive_height;
    uint16_t tile_width, tile_height;
} tsk_decode_image;

// Row table entry (parsed PREDICT tiles): word index of the row descriptor within the tile
// payload. Each tile's rows occupy one 16-byte-aligned slot of TSK_MAX_ROWS entries so that the
// slot can be staged with one bulk copy.
typedef uint16_t tsk_row_start;
#define TSK_ROW_SLOT TSK_MAX_ROWS

// Decode kernel paths a plan needs (tsk_decode_config.paths).
enum {
    TSK_PATH_U16 = 1,
    TSK_PATH_F32 = 2,
    TSK_PATH_PLAIN = 4,
    TSK_PATH_CALIBRATED = 8,
};

// Launch parameters of a decode plan: `paths` is set by the planner, the rest by
// tsk_decode_prepare (and may be lowered by the autotuner).
typedef struct {
    uint32_t grid;   // persistent CTAs: SMs x per_sm (at most the task count)
    uint32_t per_sm; // resident CTAs per SM the launch is sized for
    uint32_t smem;   // dynamic shared memory per CTA in bytes (padded so that per_sm fit exactly)
    uint32_t paths;  // TSK_PATH_* mask selecting the kernel instance
    uint32_t shape;  // plain uint16 kernel shape, 0 .. TSK_DECODE_SHAPES - 1 (decode.cu)
    uint32_t fits;   // resident CTAs per SM at the instance's occupancy
} tsk_decode_config;

// Kernel shapes of the plain uint16 decoder (consumer warps, columns per lane, stages and
// resident CTAs per SM; listed in decode.cu). Other instances map odd shapes to 0 and even
// shapes to 2.
#define TSK_DECODE_SHAPES 19

// One image to encode. 96 bytes.
typedef struct __align__(16) {
    uint64_t input;  // device address of pixel (0, 0)
    uint64_t pitch;
    uint64_t output; // device address of the .tsc file buffer
    uint64_t tile_count;
    uint64_t first_tile; // index of this image's first tile in the batch's tile sequence
    uint32_t width, height;
    uint16_t tile_width, tile_height;
    uint32_t type; // 1 = uint16, 2 = float32
    uint64_t columns;
    uint64_t reserved[3];
} tsk_encode_image;

// One standalone-calibration chunk: rows [y0, y0 + rows) of one image. 16 bytes.
typedef struct __align__(16) {
    uint32_t image;
    uint32_t y0;
    uint32_t rows;
    uint32_t reserved;
} tsk_calib_task;

// Per-image calibration state. 96 bytes.
typedef struct __align__(16) {
    uint64_t input;
    uint64_t in_pitch;
    uint64_t out;
    uint64_t out_pitch;
    uint64_t offset_map;
    uint64_t offset_pitch;
    uint64_t gain_map;
    uint64_t gain_pitch;
    float offset, gain;
    uint32_t width, height;
    uint32_t type;
    uint32_t reserved[3];
} tsk_calib_image;

// --- serving: resident archives, requests expanded into tile tasks on the device -------------

// One resident archive. Its tile templates are decode tasks with the archive-dependent fields
// set (src, words_or_tile, width, height, mode, rows_at, TSK_F32); a request fills in the rest.
typedef struct __align__(16) {
    uint64_t tiles;        // device address of tsk_decode_task[tiles_across * tiles_down]
    uint32_t tiles_across;
    uint16_t tile_width, tile_height;
    uint32_t type; // 1 = uint16, 2 = float32
    uint32_t reserved;
} tsk_serve_archive;

// One request: an ROI of one archive, written packed at out with out_pitch. 64 bytes.
typedef struct __align__(16) {
    uint64_t out;
    uint64_t out_pitch;
    uint32_t task_end; // tasks of the batch up to and including this request
    uint32_t archive;
    uint32_t x, y, width, height; // ROI in archive pixels
    uint32_t left, top, across;   // first tile column and row of the ROI; tiles per ROI row
    uint32_t flags;               // TSK_CALIBRATED or 0
    float offset, gain;           // scalar calibration
} tsk_serve_request;

// A batch of requests, passed to the kernel as its parameter block (no upload): the whole
// launch's parameters stay below the classic 4 KB limit.
#define TSK_SERVE_MAX_BATCH 48
typedef struct __align__(16) {
    uint32_t count;
    uint32_t ntasks; // requests[count - 1].task_end
    uint32_t reserved[2];
    tsk_serve_request requests[TSK_SERVE_MAX_BATCH];
} tsk_serve_batch;

// --- unparsed files: whole-image decode of .tsc files validated on the device ---------------

// One file. Its tasks (one per tile, in index order) are derived on the device; the index
// entries and row descriptors are read and validated there. image.capacity is the file size,
// image.encoder_result 0, image.tile_count the file's tiles. 192 bytes.
typedef struct __align__(16) {
    tsk_decode_image image;
    uint64_t src;         // device address of the file
    uint32_t task_end;    // tasks of the batch up to and including this file
    uint32_t tiles_across;
    uint32_t flags;       // TSK_F32 or 0
    uint32_t reserved;
    uint32_t header[16];  // the host-checked first 64 bytes the device bytes must hold
} tsk_file;

// A batch of files, passed as the kernel's parameter block (3,088 bytes: below the classic 4 KB
// limit).
#define TSK_FILE_MAX_BATCH 16
typedef struct __align__(16) {
    uint32_t count;
    uint32_t ntasks; // files[count - 1].task_end
    uint32_t reserved[2];
    tsk_file files[TSK_FILE_MAX_BATCH];
} tsk_file_batch;

// DeviceResult as seen by the kernels (types.h: {status, reserved, bytes_written}).
typedef struct {
    uint32_t status;
    uint32_t reserved;
    uint64_t bytes_written;
} tsk_result;

// --- launchers: return a cudaError_t value (0 = enqueued) ----------------------------------

// Decodes ntasks tasks. results: one record per image (the planner clears them first when
// trusted images count their completion there). claims: 4 bytes of device memory, the work
// queue's counter, which the launcher clears when the kernel shape uses it (else unused).
int tsk_decode_launch(const tsk_decode_task *tasks, uint32_t ntasks,
                      const tsk_decode_image *images, const tsk_row_start *rows,
                      tsk_result *results, tsk_decode_config config, uint32_t *claims,
                      cudaStream_t stream);
// Occupancy-derived persistent grid for a decode launch, and the kernel preload.
int tsk_decode_prepare(tsk_decode_config *config, uint32_t ntasks, int device);
// Re-sizes a prepared launch for per_sm resident CTAs per SM (at most config->fits): the grid,
// and shared memory padded so that no more CTAs share an SM.
int tsk_decode_residency(tsk_decode_config *config, uint32_t per_sm, uint32_t ntasks, int device);
// The same execution as a CUDA graph (clears of the result records when clear_results and of
// the work-queue counter when the shape uses it, then the kernel node), instantiated.
int tsk_decode_graph(const tsk_decode_task *tasks, uint32_t ntasks,
                     const tsk_decode_image *images, const tsk_row_start *rows,
                     tsk_result *results, uint32_t result_count, int clear_results,
                     tsk_decode_config config, uint32_t *claims, cudaGraph_t *graph,
                     cudaGraphExec_t *exec);

// Decodes one serving batch: tile tasks are derived from the requests and the resident archive
// templates inside the kernel. results: one record per request of the batch. all_u16: every
// archive holds uint16 samples (selects the smaller-stage kernel instance).
int tsk_serve_launch(const tsk_serve_batch *batch, const tsk_serve_archive *archives,
                     const tsk_row_start *rows, tsk_result *results, uint32_t grid, int all_u16,
                     cudaStream_t stream);
// Loads the serving kernel instance and returns its persistent grid (SMs x resident CTAs).
int tsk_serve_prepare(int all_u16, int device, uint32_t *grid);
// Decodes a batch of unparsed files (clearing their result records first, which the
// validation's completion count needs).
int tsk_file_launch(const tsk_file_batch *batch, tsk_result *results, uint32_t grid,
                    int any_f32, cudaStream_t stream);
// Loads the unparsed-file kernel instance and returns its persistent grid.
int tsk_file_prepare(int any_f32, int device, uint32_t *grid);

// Encodes every tile of every image in one pass. state: tsk_encode_state_bytes(total_tiles)
// bytes of workspace, cleared by the launcher in stream order.
int tsk_encode_launch(const tsk_encode_image *images, uint32_t image_count, uint64_t total_tiles,
                      uint32_t any_float, void *state, tsk_result *results, cudaStream_t stream);
int tsk_encode_prepare(int device);
uint64_t tsk_encode_state_bytes(uint64_t total_tiles);

// One image, scratch in a static device array (no allocation); see encode.cu.
int tsk_encode_static_launch(const tsk_encode_image *image, tsk_result *result,
                             cudaStream_t stream);
uint64_t tsk_encode_static_max_tiles(void);

// --- ROI staging: runs of bytes copied into device memory by one kernel -------------------

typedef struct {
    uint64_t src;         // device address of the run's first byte (mapped host or device memory)
    uint64_t dst;         // device address of its destination
    uint32_t bytes;       // a multiple of 4, as are src and dst
    uint32_t first_piece; // 4 KiB pieces of the runs before this one
} tsk_stage_run;

// A launch's runs, passed in the kernel parameter block (under the classic 4 KB limit).
#define TSK_STAGE_MAX_RUNS 160
typedef struct {
    uint32_t count;
    uint32_t pieces; // 4 KiB pieces of all the runs
    tsk_stage_run runs[TSK_STAGE_MAX_RUNS];
} tsk_stage_batch;

int tsk_stage_launch(const tsk_stage_batch *batch, cudaStream_t stream);

int tsk_calibrate_launch(const tsk_calib_task *tasks, uint32_t ntasks,
                         const tsk_calib_image *images, uint32_t image_count, tsk_result *results,
                         cudaStream_t stream);
int tsk_calibrate_prepare(int device);

#ifdef __cplusplus
}
#endif
