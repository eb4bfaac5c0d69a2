/*
 * TEST INFRASTRUCTURE ONLY: CPU oracle for the TileStream .tsc codec (see tsc_oracle.h).
 *
 * Plain C99 restatement of the reference CPU codec. Each function names the reference lines
 * whose behaviour it restates; status codes and the order of the checks follow the reference
 * so that every rejection maps to the same Status. Build with -O2 -ffp-contract=off.
 */
#include "tsc_oracle.h"

#include <stdlib.h>
#include <string.h>

/* L = min(INT64_MAX, SIZE_MAX) (include/tilestream/sizing.h:11-14). */
#define TSO_L ((uint64_t)(SIZE_MAX < (uint64_t)INT64_MAX ? SIZE_MAX : (uint64_t)INT64_MAX))

/* Checked arithmetic, src/checked_size.h:9-23. */
static int add_ok(uint64_t a, uint64_t b, uint64_t *r) {
    if (a > TSO_L || b > TSO_L - a) return 0;
    *r = a + b;
    return 1;
}

static int mul_ok(uint64_t a, uint64_t b, uint64_t *r) {
    if (a > TSO_L || b > TSO_L || (b != 0 && a > TSO_L / b)) return 0;
    *r = a * b;
    return 1;
}

/* src/checked_size.h:34-37: the three v1 geometries. */
static int tile_ok(uint32_t tw, uint32_t th) {
    return (tw == 128 && th == 32) || (tw == 64 && th == 64) || (tw == 256 && th == 16);
}

/* src/checked_size.h:53-62: unsupported type first, then zero dimensions. */
static int sample_size(uint32_t type, uint32_t width, uint32_t height, uint64_t *bytes) {
    if (type != TSO_UINT16 && type != TSO_FLOAT32) return TSO_UNSUPPORTED_TYPE;
    if (width == 0 || height == 0) return TSO_INVALID_ARGUMENT;
    *bytes = type == TSO_UINT16 ? 2 : 4;
    return TSO_SUCCESS;
}

static uint64_t get_le(const uint8_t *p, unsigned n) {
    uint64_t v = 0;
    for (unsigned i = 0; i < n; ++i) v |= (uint64_t)p[i] << (8 * i);
    return v;
}

static void put_le(uint8_t *p, uint64_t v, unsigned n) {
    for (unsigned i = 0; i < n; ++i) p[i] = (uint8_t)(v >> (8 * i));
}

static int all_zero(const uint8_t *p, uint64_t n) {
    for (uint64_t i = 0; i < n; ++i)
        if (p[i] != 0) return 0;
    return 1;
}

/* src/sizing.cpp:9-30. */
int tso_image_span(uint32_t type, uint32_t width, uint32_t height, uint64_t pitch,
                   uint64_t *bytes) {
    uint64_t s = 0, row = 0, span = 0;
    int st = sample_size(type, width, height, &s);
    if (st != TSO_SUCCESS) return st;
    if (!mul_ok(width, s, &row) || pitch > TSO_L) return TSO_SIZE_OVERFLOW;
    if (pitch < row || pitch % s != 0) return TSO_INVALID_ARGUMENT;
    if (!mul_ok(pitch, (uint64_t)height - 1, &span) || !add_ok(span, row, &span))
        return TSO_SIZE_OVERFLOW;
    *bytes = span;
    return TSO_SUCCESS;
}

/* src/sizing.cpp:32-59 (docs/format.md:113-134): 64 + 32 N + W H s + pad. */
int tso_compress_bound(uint32_t type, uint32_t width, uint32_t height, uint32_t tile_width,
                       uint32_t tile_height, uint64_t *bytes) {
    uint64_t s = 0, tiles = 0, index = 0, raw = 0, bound = 0;
    int st = sample_size(type, width, height, &s);
    if (st != TSO_SUCCESS) return st;
    if (!tile_ok(tile_width, tile_height)) return TSO_INVALID_ARGUMENT;
    uint64_t cols = width / tile_width + (width % tile_width != 0);
    uint64_t rows = height / tile_height + (height % tile_height != 0);
    uint64_t pad = (s == 2 && width % 2 != 0 && height % 2 != 0) ? 2 : 0;
    if (!mul_ok(cols, rows, &tiles) || !mul_ok(tiles, 32, &index) ||
        !mul_ok(width, height, &raw) || !mul_ok(raw, s, &raw) || !add_ok(64, index, &bound) ||
        !add_ok(bound, raw, &bound) || !add_ok(bound, pad, &bound))
        return TSO_SIZE_OVERFLOW;
    *bytes = bound;
    return TSO_SUCCESS;
}

/* src/cpu/views.h:9-21. */
static int byte_range(const void *data, uint64_t capacity) {
    if (capacity > TSO_L) return TSO_SIZE_OVERFLOW;
    if (data == NULL && capacity != 0) return TSO_INVALID_ARGUMENT;
    if (capacity > UINTPTR_MAX - (uintptr_t)data) return TSO_SIZE_OVERFLOW;
    return TSO_SUCCESS;
}

/* src/cpu/views.h:24-29. */
static int overlaps(const void *a, uint64_t an, const void *b, uint64_t bn) {
    uintptr_t x = (uintptr_t)a, y = (uintptr_t)b;
    return an != 0 && bn != 0 && x < y + bn && y < x + an;
}

/* src/cpu/views.h:31-46. */
static int codec_view(const void *data, uint32_t type, uint32_t width, uint32_t height,
                      uint64_t pitch, uint64_t capacity) {
    uint64_t span = 0;
    int st = tso_image_span(type, width, height, pitch, &span);
    if (st != TSO_SUCCESS) return st;
    st = byte_range(data, capacity);
    if (st != TSO_SUCCESS) return st;
    uintptr_t align = type == TSO_UINT16 ? 2 : 4;
    if (data == NULL || (uintptr_t)data % align != 0) return TSO_INVALID_ARGUMENT;
    return span <= capacity ? TSO_SUCCESS : TSO_BUFFER_TOO_SMALL;
}

/* Native table sizes counted by the reference's metadata budget (parser.cpp:173-183): on LP64
 * sizeof(ImageMetadata) = 72, sizeof(TileMetadata) = 32, sizeof(SegmentMetadata) = 24. */
static int metadata_bytes(uint64_t tiles, uint64_t segments, uint64_t *bytes) {
    uint64_t t = 0, s = 0, total = 0;
    if (!mul_ok(tiles, 32, &t) || !mul_ok(segments, 24, &s) || !add_ok(72, t, &total) ||
        !add_ok(total, s, &total))
        return TSO_SIZE_OVERFLOW;
    *bytes = total;
    return TSO_SUCCESS;
}

typedef struct {
    uint32_t type, width, height, tw, th;
    uint64_t columns, count, payload;
} header_t;

/* src/cpu/parser.cpp:27-84: the fixed header, in the reference's check order. */
static int read_header(const uint8_t *d, uint64_t size, header_t *h) {
    static const uint8_t magic[8] = {'T', 'S', 'C', 0, 13, 10, 26, 10};
    if (size < 64) return TSO_MALFORMED_DATA;
    if (memcmp(d, magic, 8) != 0) return TSO_MALFORMED_DATA;
    if (get_le(d + 8, 2) != 1 || get_le(d + 10, 2) != 0 || d[15] != 0)
        return TSO_UNSUPPORTED_FORMAT;
    if (get_le(d + 12, 2) != 64 || get_le(d + 28, 2) != 32 || !all_zero(d + 30, 2))
        return TSO_MALFORMED_DATA;
    if (d[14] != TSO_UINT16 && d[14] != TSO_FLOAT32) return TSO_UNSUPPORTED_TYPE;
    h->type = d[14];
    h->width = (uint32_t)get_le(d + 16, 4);
    h->height = (uint32_t)get_le(d + 20, 4);
    h->tw = (uint32_t)get_le(d + 24, 2);
    h->th = (uint32_t)get_le(d + 26, 2);
    if (h->width == 0 || h->height == 0) return TSO_MALFORMED_DATA;
    if (!tile_ok(h->tw, h->th)) return TSO_UNSUPPORTED_FORMAT;
    uint64_t bound = 0, index = 0;
    int st = tso_compress_bound(h->type, h->width, h->height, h->tw, h->th, &bound);
    if (st != TSO_SUCCESS) return st;
    h->columns = h->width / h->tw + (h->width % h->tw != 0);
    uint64_t rows = h->height / h->th + (h->height % h->th != 0);
    if (!mul_ok(h->columns, rows, &h->count) || !mul_ok(h->count, 32, &index) ||
        !add_ok(64, index, &h->payload))
        return TSO_SIZE_OVERFLOW;
    if (get_le(d + 32, 8) != h->count || get_le(d + 40, 8) != 64 ||
        get_le(d + 48, 8) != h->payload || get_le(d + 56, 8) != size || size > bound ||
        h->payload > size)
        return TSO_MALFORMED_DATA;
    return TSO_SUCCESS;
}

/* src/cpu/parser.cpp:86-171: validates every index entry, payload and row descriptor. With
 * tiles == NULL it only counts the row segments. */
static int walk(const uint8_t *d, uint64_t size, const header_t *h, uint64_t *segment_count,
                tso_tile *tiles, tso_segment *segments) {
    const uint64_t s = h->type == TSO_UINT16 ? 2 : 4;
    const uint32_t max_bits = h->type == TSO_UINT16 ? 16 : 32;
    uint64_t expected = h->payload, nseg = 0;
    for (uint64_t i = 0; i < h->count; ++i) {
        const uint8_t *e = d + 64 + 32 * i;
        uint64_t x = (i % h->columns) * h->tw, y = (i / h->columns) * h->th;
        uint64_t w = h->width - x < h->tw ? h->width - x : h->tw;
        uint64_t ht = h->height - y < h->th ? h->height - y : h->th;
        uint64_t off = get_le(e + 8, 8), len = get_le(e + 16, 8);
        uint64_t raw = w * ht * s, raw4 = (raw + 3) / 4 * 4;
        if (e[0] > TSO_PREDICT || !all_zero(e + 1, 3) || !all_zero(e + 24, 8) ||
            get_le(e + 4, 2) != w || get_le(e + 6, 2) != ht || off != expected || off > size ||
            len > size - off || len == 0 || len % 4 != 0 || len > raw4)
            return TSO_MALFORMED_DATA;
        const uint32_t mode = e[0];
        const uint8_t *p = d + off;
        uint64_t first = mode == TSO_PREDICT ? nseg : 0;
        if (mode == TSO_RAW) {
            if (len != raw4 || !all_zero(p + raw, len - raw)) return TSO_MALFORMED_DATA;
        } else if (mode == TSO_CONSTANT) {
            if (len != 4 || (h->type == TSO_UINT16 && !all_zero(p + 2, 2)))
                return TSO_MALFORMED_DATA;
        } else {
            uint64_t cur = 0;
            for (uint64_t r = 0; r < ht; ++r) {
                if (len - cur < 8) return TSO_MALFORMED_DATA;
                const uint8_t *desc = p + cur;
                uint32_t seed = (uint32_t)get_le(desc, 4);
                uint32_t bits = desc[4];
                if ((h->type == TSO_UINT16 && seed > 0xffffu) || bits > max_bits ||
                    (w == 1 && bits != 0) || !all_zero(desc + 5, 3))
                    return TSO_MALFORMED_DATA;
                cur += 8;
                uint64_t nbits = (w - 1) * bits, packed = (nbits + 31) / 32 * 4;
                if (packed > len - cur) return TSO_MALFORMED_DATA;
                if (nbits % 32 != 0) {
                    uint32_t last = (uint32_t)get_le(p + cur + packed - 4, 4);
                    if ((last >> (nbits % 32)) != 0) return TSO_MALFORMED_DATA;
                }
                if (segments != NULL) {
                    segments[nseg].seed = seed;
                    segments[nseg].bit_width = bits;
                    segments[nseg].payload_offset = cur;
                    segments[nseg].payload_bytes = packed;
                }
                ++nseg;
                cur += packed;
            }
            if (cur != len) return TSO_MALFORMED_DATA;
        }
        if (tiles != NULL) {
            tiles[i].mode = mode;
            tiles[i].width = (uint16_t)w;
            tiles[i].height = (uint16_t)ht;
            tiles[i].offset = off;
            tiles[i].length = len;
            tiles[i].first_segment = first;
        }
        expected += len;
    }
    *segment_count = nseg;
    return expected == size ? TSO_SUCCESS : TSO_MALFORMED_DATA;
}

/* src/cpu/parser.cpp:187-223 (everything up to the allocation of the tables). */
int tso_parse_layout(const uint8_t *file, uint64_t size, const tso_limits *limits,
                     tso_layout *layout) {
    tso_limits none = {TSO_L, TSO_L, TSO_L};
    const tso_limits *lim = limits != NULL ? limits : &none;
    header_t h;
    uint64_t need = 0, nseg = 0;
    int st = byte_range(file, size);
    if (st != TSO_SUCCESS) return st;
    if (size > lim->file_bytes) return TSO_RESOURCE_LIMIT;
    st = read_header(file, size, &h);
    if (st != TSO_SUCCESS) return st;
    if (h.count > lim->tile_count) return TSO_RESOURCE_LIMIT;
    st = metadata_bytes(h.count, 0, &need);
    if (st != TSO_SUCCESS) return st;
    if (need > lim->metadata_bytes) return TSO_RESOURCE_LIMIT;
    st = walk(file, size, &h, &nseg, NULL, NULL);
    if (st != TSO_SUCCESS) return st;
    st = metadata_bytes(h.count, nseg, &need);
    if (st != TSO_SUCCESS) return st;
    if (need > lim->metadata_bytes) return TSO_RESOURCE_LIMIT;
    layout->type = h.type;
    layout->width = h.width;
    layout->height = h.height;
    layout->tile_width = (uint16_t)h.tw;
    layout->tile_height = (uint16_t)h.th;
    layout->file_bytes = size;
    layout->tile_count = h.count;
    layout->segment_count = nseg;
    return TSO_SUCCESS;
}

/* src/cpu/parser.cpp:224-236: the second walk fills the tables. */
int tso_parse_fill(const uint8_t *file, uint64_t size, const tso_layout *layout, tso_tile *tiles,
                   tso_segment *segments) {
    header_t h;
    uint64_t nseg = 0;
    int st = read_header(file, size, &h);
    if (st != TSO_SUCCESS) return st;
    if (h.count != layout->tile_count) return TSO_INVALID_ARGUMENT;
    return walk(file, size, &h, &nseg, tiles, segments);
}

/* src/cpu/decoder.cpp:11-27: residual j of a row of b-bit symbols. A second word is read only
 * when the symbol crosses into it; b = 0 and b = 32 are explicit (docs/format.md:79). */
static uint32_t symbol(const uint8_t *packed, uint32_t j, uint32_t b) {
    if (b == 0) return 0;
    if (b == 32) return (uint32_t)get_le(packed + 4 * (uint64_t)j, 4);
    uint64_t pos = (uint64_t)j * b;
    uint32_t shift = (uint32_t)(pos % 32);
    const uint8_t *w = packed + (pos / 32) * 4;
    uint32_t v = (uint32_t)get_le(w, 4) >> shift;
    if (shift + b > 32) v |= (uint32_t)get_le(w + 4, 4) << (32 - shift);
    return v & ((1u << b) - 1);
}

/* src/cpu/decoder.cpp:29-82: pixel reconstruction from validated metadata. */
static void reconstruct(const uint8_t *file, const tso_layout *L, const tso_tile *tiles,
                        const tso_segment *segs, uint8_t *out, uint64_t pitch) {
    const uint64_t s = L->type == TSO_UINT16 ? 2 : 4;
    const uint64_t cols = L->width / L->tile_width + (L->width % L->tile_width != 0);
    for (uint64_t i = 0; i < L->tile_count; ++i) {
        const tso_tile *t = &tiles[i];
        uint64_t x = (i % cols) * L->tile_width, y = (i / cols) * L->tile_height;
        const uint8_t *p = file + t->offset;
        for (uint32_t r = 0; r < t->height; ++r) {
            uint8_t *line = out + (y + r) * pitch + x * s;
            if (t->mode == TSO_RAW) {
                memcpy(line, p + (uint64_t)r * t->width * s, t->width * s);
            } else if (t->mode == TSO_CONSTANT) {
                uint32_t v = (uint32_t)get_le(p, 4);
                for (uint32_t c = 0; c < t->width; ++c) put_le(line + c * s, v, (unsigned)s);
            } else {
                const tso_segment *g = &segs[t->first_segment + r];
                uint32_t prev = g->seed;
                put_le(line, prev, (unsigned)s);
                for (uint32_t c = 1; c < t->width; ++c) {
                    uint32_t z = symbol(p + g->payload_offset, c - 1, g->bit_width);
                    if (L->type == TSO_UINT16) {
                        /* Inverse zigzag, then add modulo 2^16 (docs/format.md:81-93). */
                        int32_t delta = (z & 1u) ? -(int32_t)(z >> 1) - 1 : (int32_t)(z >> 1);
                        prev = (uint32_t)((int32_t)prev + delta) & 0xffffu;
                    } else {
                        prev ^= z; /* docs/format.md:95-97 */
                    }
                    put_le(line + c * s, prev, (unsigned)s);
                }
            }
        }
    }
}

/* src/cpu/decoder.cpp:86-110. */
int tso_decompress(const uint8_t *file, uint64_t size, void *pixels, uint32_t type,
                   uint32_t width, uint32_t height, uint64_t pitch, uint64_t capacity,
                   const tso_limits *limits) {
    tso_layout L;
    int st = codec_view(pixels, type, width, height, pitch, capacity);
    if (st != TSO_SUCCESS) return st;
    st = byte_range(file, size);
    if (st != TSO_SUCCESS) return st;
    if (overlaps(file, size, pixels, capacity)) return TSO_INVALID_ARGUMENT;
    st = tso_parse_layout(file, size, limits, &L);
    if (st != TSO_SUCCESS) return st;
    tso_tile *tiles = (tso_tile *)malloc((L.tile_count ? L.tile_count : 1) * sizeof(tso_tile));
    tso_segment *segs =
        (tso_segment *)malloc((L.segment_count ? L.segment_count : 1) * sizeof(tso_segment));
    if (tiles == NULL || segs == NULL) {
        free(tiles);
        free(segs);
        return TSO_RESOURCE_LIMIT;
    }
    st = tso_parse_fill(file, size, &L, tiles, segs);
    if (st == TSO_SUCCESS &&
        (width != L.width || height != L.height || type != L.type))
        st = TSO_INVALID_ARGUMENT;
    if (st == TSO_SUCCESS) reconstruct(file, &L, tiles, segs, (uint8_t *)pixels, pitch);
    free(tiles);
    free(segs);
    return st;
}

/* src/cpu/encoder.cpp:32-37: zigzag of the signed difference modulo 2^16. */
static uint32_t zigzag16(uint32_t cur, uint32_t prev) {
    uint32_t d = (cur - prev) & 0xffffu;
    int32_t sd = d < 32768u ? (int32_t)d : (int32_t)d - 65536;
    return sd >= 0 ? (uint32_t)(2 * sd) : (uint32_t)(-2 * sd - 1);
}

typedef struct {
    uint32_t samples[4096];
    uint32_t residuals[4096];
    uint32_t widths[64];
    uint32_t mode;
    uint64_t length;
} tile_plan;

/* src/cpu/encoder.cpp:39-79: residuals, minimal row widths and the canonical mode choice
 * RAW < CONSTANT < PREDICT_BITPACK on ties (docs/format.md:99-109). */
static void analyze(const uint8_t *base, uint32_t type, uint64_t pitch, uint64_t x, uint64_t y,
                    uint32_t w, uint32_t h, tile_plan *t) {
    const uint64_t s = type == TSO_UINT16 ? 2 : 4;
    int constant = 1;
    uint64_t predictive = 0;
    for (uint32_t r = 0; r < h; ++r) {
        uint32_t or_all = 0;
        for (uint32_t c = 0; c < w; ++c) {
            uint32_t k = r * w + c;
            t->samples[k] = (uint32_t)get_le(base + (y + r) * pitch + (x + c) * s, (unsigned)s);
            constant = constant && t->samples[k] == t->samples[0];
            if (c != 0) {
                uint32_t z = type == TSO_UINT16 ? zigzag16(t->samples[k], t->samples[k - 1])
                                                : t->samples[k] ^ t->samples[k - 1];
                t->residuals[k] = z;
                or_all |= z;
            }
        }
        uint32_t bits = 0;
        while (or_all != 0) {
            ++bits;
            or_all >>= 1;
        }
        t->widths[r] = bits;
        predictive += 8 + (((uint64_t)(w - 1) * bits + 31) / 32) * 4;
    }
    t->mode = TSO_RAW;
    t->length = ((uint64_t)w * h * s + 3) / 4 * 4;
    if (constant && 4 < t->length) {
        t->mode = TSO_CONSTANT;
        t->length = 4;
    }
    if (predictive < t->length) {
        t->mode = TSO_PREDICT;
        t->length = predictive;
    }
}

/* src/cpu/encoder.cpp:81-118: payload bytes of one tile, zero padded. Residuals are packed
 * least significant bit first with a 64-bit accumulator; the bit positions are the same as the
 * reference's bit-by-bit loop (docs/format.md:77). */
static void write_payload(uint8_t *out, const tile_plan *t, uint32_t type, uint32_t w,
                          uint32_t h) {
    memset(out, 0, (size_t)t->length);
    const unsigned s = type == TSO_UINT16 ? 2 : 4;
    if (t->mode == TSO_RAW) {
        for (uint32_t i = 0; i < w * h; ++i) put_le(out + (uint64_t)i * s, t->samples[i], s);
    } else if (t->mode == TSO_CONSTANT) {
        put_le(out, t->samples[0], s);
    } else {
        for (uint32_t r = 0; r < h; ++r) {
            uint32_t b = t->widths[r];
            put_le(out, t->samples[r * w], 4);
            out[4] = (uint8_t)b;
            out += 8;
            uint64_t acc = 0;
            unsigned have = 0;
            uint8_t *dst = out;
            for (uint32_t c = 1; c < w; ++c) {
                acc |= (uint64_t)t->residuals[r * w + c] << have;
                have += b;
                while (have >= 32) {
                    put_le(dst, (uint32_t)acc, 4);
                    dst += 4;
                    acc >>= 32;
                    have -= 32;
                }
            }
            if (have > 0) put_le(dst, (uint32_t)acc, 4);
            out += (((uint64_t)(w - 1) * b + 31) / 32) * 4;
        }
    }
}

/* src/cpu/encoder.cpp:120-140. */
static void write_header(uint8_t *o, uint32_t type, uint32_t width, uint32_t height,
                         uint32_t tw, uint32_t th, uint64_t count, uint64_t length) {
    static const uint8_t magic[8] = {'T', 'S', 'C', 0, 13, 10, 26, 10};
    memset(o, 0, 64);
    memcpy(o, magic, 8);
    put_le(o + 8, 1, 2);
    put_le(o + 10, 0, 2);
    put_le(o + 12, 64, 2);
    o[14] = (uint8_t)type;
    put_le(o + 16, width, 4);
    put_le(o + 20, height, 4);
    put_le(o + 24, tw, 2);
    put_le(o + 26, th, 2);
    put_le(o + 28, 32, 2);
    put_le(o + 32, count, 8);
    put_le(o + 40, 64, 8);
    put_le(o + 48, 64 + count * 32, 8);
    put_le(o + 56, length, 8);
}

/* src/cpu/encoder.cpp:144-197. */
int tso_compress(const void *pixels, uint32_t type, uint32_t width, uint32_t height,
                 uint64_t pitch, uint64_t capacity, uint32_t tile_width, uint32_t tile_height,
                 uint8_t *out, uint64_t out_size, uint64_t *written) {
    uint64_t bound = 0;
    int st = codec_view(pixels, type, width, height, pitch, capacity);
    if (st != TSO_SUCCESS) return st;
    st = tso_compress_bound(type, width, height, tile_width, tile_height, &bound);
    if (st != TSO_SUCCESS) return st;
    st = byte_range(out, out_size);
    if (st != TSO_SUCCESS) return st;
    if (out_size < bound) return TSO_BUFFER_TOO_SMALL;
    if (overlaps(pixels, capacity, out, out_size) ||
        overlaps(written, sizeof(*written), out, out_size) ||
        overlaps(written, sizeof(*written), pixels, capacity))
        return TSO_INVALID_ARGUMENT;
    const uint64_t cols = width / tile_width + (width % tile_width != 0);
    const uint64_t rows = height / tile_height + (height % tile_height != 0);
    const uint64_t count = cols * rows;
    uint64_t cursor = 64 + count * 32;
    tile_plan *t = (tile_plan *)malloc(sizeof(tile_plan));
    if (t == NULL) return TSO_RESOURCE_LIMIT;
    for (uint64_t i = 0; i < count; ++i) {
        uint64_t x = (i % cols) * tile_width, y = (i / cols) * tile_height;
        uint32_t w = (uint32_t)(width - x < tile_width ? width - x : tile_width);
        uint32_t h = (uint32_t)(height - y < tile_height ? height - y : tile_height);
        analyze((const uint8_t *)pixels, type, pitch, x, y, w, h, t);
        uint8_t *e = out + 64 + i * 32;
        memset(e, 0, 32);
        e[0] = (uint8_t)t->mode;
        put_le(e + 4, w, 2);
        put_le(e + 6, h, 2);
        put_le(e + 8, cursor, 8);
        put_le(e + 16, t->length, 8);
        write_payload(out + cursor, t, type, w, h);
        cursor += t->length;
    }
    free(t);
    write_header(out, type, width, height, tile_width, tile_height, count, cursor);
    *written = cursor;
    return TSO_SUCCESS;
}

/* tests/numerics/support.h:34-38 and src/cuda/device.cuh:81-85: RN(RN(x - offset) * gain). */
float tso_calibrate(float x, float offset, float gain) {
    volatile float difference = x - offset;
    return difference * gain;
}

/* tests/numerics/support.h:40-44. */
double tso_calibrate_f64(float x, float offset, float gain) {
    double difference = (double)x - (double)offset;
    return difference * (double)gain;
}

void tso_calibrate_image(const void *input, uint32_t type, uint32_t width, uint32_t height,
                         uint64_t in_pitch, float offset, const float *offset_map,
                         uint64_t offset_pitch, float gain, const float *gain_map,
                         uint64_t gain_pitch, float *output, uint64_t out_pitch) {
    for (uint32_t y = 0; y < height; ++y) {
        const uint8_t *row = (const uint8_t *)input + y * in_pitch;
        float *dst = (float *)((uint8_t *)output + y * out_pitch);
        const float *om = offset_map ? (const float *)((const uint8_t *)offset_map +
                                                       y * offset_pitch)
                                     : NULL;
        const float *gm =
            gain_map ? (const float *)((const uint8_t *)gain_map + y * gain_pitch) : NULL;
        for (uint32_t x = 0; x < width; ++x) {
            float v;
            if (type == TSO_UINT16) {
                v = (float)get_le(row + 2 * (uint64_t)x, 2);
            } else {
                uint32_t bits = (uint32_t)get_le(row + 4 * (uint64_t)x, 4);
                memcpy(&v, &bits, 4);
            }
            dst[x] = tso_calibrate(v, om ? om[x] : offset, gm ? gm[x] : gain);
        }
    }
}
