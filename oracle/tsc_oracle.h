/*
 * TEST INFRASTRUCTURE ONLY: the CPU oracle for the TileStream .tsc codec path.
 *
 * A plain-C restatement of the reference CPU codec (src/cpu/{parser,encoder,decoder}.cpp,
 * src/sizing.cpp) and of the host calibration forms (tests/numerics/support.h:34-44). It is the
 * checker that the CUDA path is compared against. Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline / reference legs may load it; no product code links it.
 *
 * Parity pinned: tests/test_oracle.py checks this oracle byte-for-byte against the 8
 * hand-calculated golden files (the .hex files in tests/golden, produced by the reference encoder itself by
 * tests/golden/make_golden.py) and against the reference CPU codec compiled from its own sources
 * into oracle/_ref (oracle/Makefile) on the seeded robustness cases and the C1 frame.
 *
 * Status values are the reference's Status enum (include/tilestream/types.h:7-19).
 */
#ifndef TSC_ORACLE_H
#define TSC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    TSO_SUCCESS = 0,
    TSO_INVALID_ARGUMENT = 1,
    TSO_INVALID_ROI = 2,
    TSO_UNSUPPORTED_TYPE = 3,
    TSO_UNSUPPORTED_FORMAT = 4,
    TSO_MALFORMED_DATA = 5,
    TSO_SIZE_OVERFLOW = 6,
    TSO_BUFFER_TOO_SMALL = 7,
    TSO_RESOURCE_LIMIT = 8,
};

enum { TSO_UINT16 = 1, TSO_FLOAT32 = 2 };
enum { TSO_RAW = 0, TSO_CONSTANT = 1, TSO_PREDICT = 2 };

/* Same layout as tilestream::TileMetadata (32 B) and SegmentMetadata (24 B). */
typedef struct {
    uint32_t mode;
    uint16_t width;
    uint16_t height;
    uint64_t offset;
    uint64_t length;
    uint64_t first_segment;
} tso_tile;

typedef struct {
    uint32_t seed;
    uint32_t bit_width;
    uint64_t payload_offset;
    uint64_t payload_bytes;
} tso_segment;

typedef struct {
    uint32_t type;
    uint32_t width;
    uint32_t height;
    uint16_t tile_width;
    uint16_t tile_height;
    uint64_t file_bytes;
    uint64_t tile_count;
    uint64_t segment_count;
} tso_layout;

typedef struct {
    uint64_t file_bytes;
    uint64_t tile_count;
    uint64_t metadata_bytes;
} tso_limits;

/* Size queries: src/sizing.cpp:9-30 and :32-59. */
int tso_image_span(uint32_t type, uint32_t width, uint32_t height, uint64_t pitch,
                   uint64_t *bytes);
int tso_compress_bound(uint32_t type, uint32_t width, uint32_t height, uint32_t tile_width,
                       uint32_t tile_height, uint64_t *bytes);

/* Parser pass 1 (header + counting walk) and pass 2 (fill): src/cpu/parser.cpp:187-242.
 * limits may be NULL for "no budget". */
int tso_parse_layout(const uint8_t *file, uint64_t size, const tso_limits *limits,
                     tso_layout *layout);
int tso_parse_fill(const uint8_t *file, uint64_t size, const tso_layout *layout, tso_tile *tiles,
                   tso_segment *segments);

/* Whole-file decode into a pitched image: src/cpu/decoder.cpp:86-110. */
int tso_decompress(const uint8_t *file, uint64_t size, void *pixels, uint32_t type,
                   uint32_t width, uint32_t height, uint64_t pitch, uint64_t capacity,
                   const tso_limits *limits);

/* Canonical encode: src/cpu/encoder.cpp:144-197. */
int tso_compress(const void *pixels, uint32_t type, uint32_t width, uint32_t height,
                 uint64_t pitch, uint64_t capacity, uint32_t tile_width, uint32_t tile_height,
                 uint8_t *out, uint64_t out_size, uint64_t *written);

/* Host calibration forms: tests/numerics/support.h:34-44 (two binary32 roundings, and the
 * FP64 reference). The file is compiled with -ffp-contract=off. */
float tso_calibrate(float x, float offset, float gain);
double tso_calibrate_f64(float x, float offset, float gain);

/* Calibrates a whole pitched image of samples (uint16 or FP32 words). offset_map / gain_map
 * may be NULL to use the scalars; maps are FP32 images in output coordinates. */
void tso_calibrate_image(const void *input, uint32_t type, uint32_t width, uint32_t height,
                         uint64_t in_pitch, float offset, const float *offset_map,
                         uint64_t offset_pitch, float gain, const float *gain_map,
                         uint64_t gain_pitch, float *output, uint64_t out_pitch);

#ifdef __cplusplus
}
#endif

#endif
