// Single-launch canonical .tsc encoder for sm_100a.
//
// The reference encodes a window with four launches and a library scan: analyze (residuals to
// a 16 KiB-per-tile global workspace), cub::DeviceScan over tile lengths, pack (re-reading the
// input and the residuals) and finish (src/cuda/encoder.cu:62-327). Here one persistent kernel
// does all of it:
//
//  1. a CTA claims the next chunk of k consecutive tiles (in batch order, from an atomic
//     counter; k = ceil(tiles / grid), at most half the shared-memory payload slots: 2 uint16
//     or 1 FP32 tile) and, tile by tile, copies the pixels into shared memory (16-byte cp.async,
//     the next tile in flight while the current one is encoded). Each thread takes a 16-sample
//     segment of a row and computes its residuals in registers (zigzag mod 2^16 or XOR,
//     encoder.cpp:32-37); the row width is the index of the highest set bit of the row's OR
//     (docs/format.md:101), the row costs are scanned with a warp shuffle scan, and the canonical
//     mode is chosen with the tie order RAW < CONSTANT < PREDICT (docs/format.md:103-109,
//     encoder.cpp:69-78). The tile is then encoded into its payload slot in shared memory: each
//     thread appends its residuals to the row's bit stream;
//  2. the chunk publishes the summed lengths of its tiles of its last image, in its own word and
//     added (with an arrival count) to the word of its group of 32 chunks. Its offsets need the
//     lengths of the earlier chunks of its first image: whole groups from their group words, the
//     chunks at either end from their own words. Each word read is final as soon as the chunks it
//     covers are encoded, so a look-back never waits for another look-back (a chain of inclusive
//     prefixes advances one window per L2 round trip; a look-back per tile would wait on many
//     more chunks). The CTA reads them one chunk later, while it encodes its next chunk: every
//     thread has one word in flight during that chunk's first tile. Waits are bounded and report
//     cuda_error instead of hanging;
//  3. the CTA writes the index entries and copies the payloads out, each word by exactly one
//     thread (the reference's pack gathers the same bits from global memory,
//     encoder.cu:157-173), a tile of the previous chunk beside each tile of the next one, so the
//     stores spread over the encoding instead of arriving all at once;
//  4. the last tile of an image writes the 64-byte header and the image's DeviceResult.
#include "ptx.cuh"
#include "tasks.h"

#include <cstdint>
#include <mutex>

namespace tsk {
namespace {

constexpr uint32_t kThreads = 256;
// A chunk's word: kPublished | the summed lengths. A group's word: the number of its chunks that
// have added their lengths, in the top byte, and the sum of those lengths.
constexpr uint64_t kPublished = 1ull << 62;
constexpr uint64_t kValue = (1ull << 62) - 1;
constexpr uint32_t kGroupChunks = 32;
constexpr uint64_t kGroupArrival = 1ull << 56;
constexpr uint64_t kGroupValue = kGroupArrival - 1;

constexpr uint32_t kMaxChunk = 2; // tiles per chunk: half the payload slots

// Divides small numerators (n * d < 2^32) by d with a multiply: floor(n / d) equals the high
// word of n * ceil(2^32 / d).
struct Divider {
    uint32_t d, magic;
    __device__ static Divider of(uint32_t d) {
        return {d, d > 1 ? 0xffffffffu / d + 1u : 0u};
    }
    __device__ __forceinline__ uint32_t div(uint32_t n) const {
        return d > 1 ? __umulhi(n, magic) : n;
    }
};

// One tile of a chunk, computed once when the chunk is claimed: its position in its image and
// the divisors of its copy and segment layouts.
struct TileGeom {
    uint64_t x, y;
    uint64_t index;  // tile index within its image
    uint64_t origin; // address of the tile's pixel (0, 0)
    uint32_t w, h;
    uint32_t vector; // rows are 16-byte multiples at 16-byte-aligned addresses
    Divider vec_per_row; // 16-byte pieces per row (when rows are 16-byte multiples)
    Divider seg_per_row; // thread segments per row
};

// A claimed chunk: tiles [first, first + count) of the batch, and what is known of them.
struct Chunk {
    uint64_t id;
    uint64_t first;
    uint32_t count;
    uint32_t slot0;            // payload slot of its first tile
    uint64_t carry;            // lengths of its first image's tiles in earlier chunks
    uint64_t stop;             // the chunk holding its first image's first tile
    uint32_t image[kMaxChunk]; // image of each tile of the chunk
    TileGeom geom[kMaxChunk];
    uint32_t mode_of[kMaxChunk];
    uint32_t length_of[kMaxChunk];
    uint64_t offset[kMaxChunk]; // payload offset within its image's payload area, less the carry
};

// Words: the largest tile in 32-bit words, 2048 for uint16-only batches (4096 samples) and
// 4096 when the batch has FP32 images; a PREDICT payload is always shorter than the RAW one.
// Slots: payloads kept until their offsets are known, for two chunks (the one being encoded
// and the one before it, written out meanwhile).
template <uint32_t Words, uint32_t Slots> struct EncodeShared {
    static constexpr uint32_t kSlots = Slots;
    // Two tile buffers: the tile being analysed and the next one in flight. Rows are packed
    // (w samples each), as uint16 or FP32 words.
    alignas(16) uint32_t raw[2][Words];
    alignas(16) uint32_t payload[Slots][Words]; // encoded payloads of the two chunks
    uint32_t row_or[TSK_MAX_ROWS];         // OR of each row's residuals
    uint32_t bits[TSK_MAX_ROWS];
    uint32_t row_word[TSK_MAX_ROWS + 1]; // first payload word of each row
    uint32_t mode;
    uint32_t length;
    // The chunk being encoded, the one before it and the next one, in rotation.
    Chunk chunks[3];
};

// Residual of a sample against its left neighbour: for uint16 the zigzag of the difference
// taken as a signed 16-bit value, 2d for d >= 0 and -2d - 1 for d < 0 (encoder.cpp:32-37); for
// FP32 words the XOR of the bit patterns.
template <bool F32> __device__ __forceinline__ uint32_t residual(uint32_t cur, uint32_t prev) {
    if constexpr (F32) {
        return cur ^ prev;
    } else {
        const int32_t d = static_cast<int16_t>(static_cast<uint16_t>(cur - prev));
        return static_cast<uint32_t>((d * 2) ^ (d >> 31));
    }
}

// Look-back words carry their own values (nothing else is read on the strength of one), so
// relaxed device-scope accesses suffice; a relaxed load does not hold back the loads after it.
__device__ __forceinline__ uint64_t ld_relaxed(const uint64_t *p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_relaxed(uint64_t *p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void put_word(uint8_t *file, uint64_t byte, uint32_t v) {
    *reinterpret_cast<uint32_t *>(file + byte) = v;
}

__device__ TileGeom tile_geom(const tsk_encode_image &im, uint64_t index) {
    TileGeom g;
    g.index = index;
    g.x = (index % im.columns) * im.tile_width;
    g.y = (index / im.columns) * im.tile_height;
    g.w = static_cast<uint32_t>(im.width - g.x < im.tile_width ? im.width - g.x : im.tile_width);
    g.h = static_cast<uint32_t>(im.height - g.y < im.tile_height ? im.height - g.y
                                                                 : im.tile_height);
    const uint32_t s = im.type == 2 ? 4 : 2;
    g.origin = im.input + g.y * im.pitch + g.x * s;
    g.vector = ((g.origin | im.pitch | (g.w * s)) & 15u) == 0;
    g.vec_per_row = Divider::of((g.w * s) / 16 != 0 ? (g.w * s) / 16 : 1);
    g.seg_per_row = Divider::of((g.w + 15) / 16);
    return g;
}

// Sample i of the tile in buffer `buf` (rows packed, w samples each).
template <bool F32, typename Sh>
__device__ __forceinline__ uint32_t px(const Sh &sh, uint32_t buf, uint32_t i) {
    if constexpr (F32) {
        return sh.raw[buf][i];
    } else {
        return reinterpret_cast<const uint16_t *>(sh.raw[buf])[i];
    }
}

// Starts copying the tile's pixels into buffer `buf` and closes this thread's cp.async group.
// Rows whose bytes are a multiple of 16 at 16-byte-aligned addresses go as 16-byte cp.async
// copies issued by the whole CTA at once; other tiles are copied synchronously.
template <bool F32, typename Sh>
__device__ void issue_tile(Sh &sh, uint32_t buf, const tsk_encode_image &im, const TileGeom &g) {
    constexpr uint32_t s = F32 ? 4 : 2;
    const uint32_t w = g.w, h = g.h;
    const uint32_t row_bytes = w * s;
    const uint8_t *origin = reinterpret_cast<const uint8_t *>(g.origin);
    uint8_t *dst = reinterpret_cast<uint8_t *>(sh.raw[buf]);
    if (g.vector != 0) {
        const uint32_t per_row = row_bytes / 16;
        for (uint32_t c = threadIdx.x; c < h * per_row; c += kThreads) {
            const uint32_t r = g.vec_per_row.div(c), k = c - r * per_row;
            cp_async16(dst + r * row_bytes + 16 * k, origin + r * im.pitch + 16 * k);
        }
    } else {
        for (uint32_t i = threadIdx.x; i < w * h; i += kThreads) {
            const uint32_t r = i / w, c = i - r * w;
            const uint8_t *line = origin + r * im.pitch;
            if constexpr (F32) {
                sh.raw[buf][i] = reinterpret_cast<const uint32_t *>(line)[c];
            } else {
                reinterpret_cast<uint16_t *>(sh.raw[buf])[i] =
                    reinterpret_cast<const uint16_t *>(line)[c];
            }
        }
    }
    cp_async_commit();
}

template <bool AnyF32, typename Sh>
__device__ __forceinline__ void issue_tile_any(Sh &sh, uint32_t buf, const tsk_encode_image &im,
                                               const TileGeom &g) {
    if (AnyF32 && im.type == 2) {
        issue_tile<true>(sh, buf, im, g);
    } else {
        issue_tile<false>(sh, buf, im, g);
    }
}

// This thread's part of a tile: kSeg consecutive samples of one row.
constexpr uint32_t kSeg = 16;

struct Segment {
    uint32_t r, c0, n; // row, first column, samples (n = 0: no part)
};

__device__ __forceinline__ Segment segment_of(const TileGeom &g) {
    const uint32_t per_row = g.seg_per_row.d;
    Segment seg{0, 0, 0};
    if (threadIdx.x < per_row * g.h) {
        seg.r = g.seg_per_row.div(threadIdx.x);
        seg.c0 = (threadIdx.x - seg.r * per_row) * kSeg;
        seg.n = g.w - seg.c0 < kSeg ? g.w - seg.c0 : kSeg;
    }
    return seg;
}

// The segment's residuals z[k] (column c0 + k; zero for column 0 and past the segment), their
// OR, and its first sample.
template <bool F32, typename Sh>
__device__ __forceinline__ void segment_residuals(const Sh &sh, uint32_t buf,
                                                  const TileGeom &g, const Segment &seg,
                                                  uint32_t (&z)[kSeg], uint32_t &orv,
                                                  uint32_t &head) {
    const uint32_t base = seg.r * g.w + seg.c0;
    uint32_t x[kSeg];
    // A whole segment of a row that starts on 16 bytes is read with 16-byte loads (neighbouring
    // threads' segments are 32 or 64 bytes apart, so sample-by-sample reads conflict on banks).
    constexpr uint32_t kPerVec = F32 ? 4 : 8;
    if (seg.n == kSeg && g.w % kPerVec == 0) {
        const uint4 *v = reinterpret_cast<const uint4 *>(sh.raw[buf]) + base / kPerVec;
#pragma unroll
        for (uint32_t q = 0; q < kSeg / kPerVec; ++q) {
            const uint4 u = v[q];
            if constexpr (F32) {
                x[4 * q] = u.x;
                x[4 * q + 1] = u.y;
                x[4 * q + 2] = u.z;
                x[4 * q + 3] = u.w;
            } else {
                const uint32_t wd[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
                for (uint32_t e = 0; e < 4; ++e) {
                    x[8 * q + 2 * e] = wd[e] & 0xffffu;
                    x[8 * q + 2 * e + 1] = wd[e] >> 16;
                }
            }
        }
    } else {
#pragma unroll
        for (uint32_t k = 0; k < kSeg; ++k) {
            // Past the segment the last sample repeats, so the residual is zero.
            x[k] = px<F32>(sh, buf, base + (k < seg.n ? k : seg.n - 1));
        }
    }
    uint32_t prev = seg.c0 > 0 ? px<F32>(sh, buf, base - 1) : x[0];
    head = x[0];
    orv = 0;
#pragma unroll
    for (uint32_t k = 0; k < kSeg; ++k) {
        z[k] = residual<F32>(x[k], prev); // column 0 compares the sample with itself: zero
        orv |= z[k];
        prev = x[k];
    }
}

// Row widths, the constant test, the row-cost scan and the canonical mode; sets sh.bits,
// sh.row_word, sh.mode and sh.length. z keeps the segment's residuals for pack_tile.
template <bool F32, typename Sh>
__device__ void analyze_tile(Sh &sh, uint32_t buf, const TileGeom &g,
                             const Segment &seg, uint32_t (&z)[kSeg]) {
    const uint32_t warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    constexpr uint32_t s = F32 ? 4 : 2;
    const uint32_t w = g.w, h = g.h;
    // The tile is constant when every row starts with the tile's first sample and no row has a
    // nonzero residual.
    uint32_t orv = 0, head = 0;
    bool seed_ok = true;
    if (seg.n != 0) {
        segment_residuals<F32>(sh, buf, g, seg, z, orv, head);
        if (orv != 0) {
            atomicOr(&sh.row_or[seg.r], orv);
        }
        seed_ok = seg.c0 != 0 || head == px<F32>(sh, buf, 0);
    }
    bool uniform = __syncthreads_and(seed_ok) != 0;

    // Row costs in words (descriptor + packed residuals), scanned by warp 0.
    if (warp == 0) {
        uint32_t carry = 0;
        for (uint32_t base = 0; base < h; base += 32) {
            const uint32_t r = base + lane;
            uint32_t cost = 0;
            if (r < h) {
                const uint32_t b = 32u - __clz(sh.row_or[r]);
                sh.bits[r] = b;
                cost = 2u + ((w - 1) * b + 31u) / 32u;
            }
            uniform = __all_sync(0xffffffffu, uniform && (r >= h || sh.row_or[r] == 0));
            uint32_t incl = cost;
#pragma unroll
            for (uint32_t d = 1; d < 32; d <<= 1) {
                const uint32_t o = __shfl_up_sync(0xffffffffu, incl, d);
                if (lane >= d) incl += o;
            }
            if (r < h) {
                sh.row_word[r] = carry + incl - cost;
            }
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (lane == 0) {
            sh.row_word[h] = carry;
            // Canonical choice (docs/format.md:103-109).
            uint32_t mode = TSK_RAW;
            uint32_t length = (w * h * s + 3u) / 4u * 4u;
            if (uniform && 4u < length) {
                mode = TSK_CONSTANT;
                length = 4;
            }
            if (4u * carry < length) {
                mode = TSK_PREDICT;
                length = 4u * carry;
            }
            sh.mode = mode;
            sh.length = length;
        }
    }
    __syncthreads();
}

// Encodes an analysed tile into payload slot `slot`. PREDICT rows: each thread appends its
// segment's residuals to the row's bit stream (docs/format.md:77) through a 64-bit accumulator,
// OR-ing the words it touches into the slot (cleared before the tile's first barrier). RAW: the
// tile buffer holds the rows packed, so it is copied, zero-padded to a word. CONSTANT: one word.
template <bool F32, typename Sh>
__device__ void pack_tile(Sh &sh, uint32_t buf, uint32_t slot, const TileGeom &g,
                          const Segment &seg, const uint32_t (&z)[kSeg]) {
    const uint32_t w = g.w, h = g.h;
    const uint32_t mode = sh.mode, words = sh.length / 4;
    uint32_t *out = sh.payload[slot];
    if (mode == TSK_RAW) {
        const uint32_t bytes = w * h * (F32 ? 4 : 2);
        for (uint32_t k = threadIdx.x; k < words; k += kThreads) {
            uint32_t v = sh.raw[buf][k];
            if (4 * k + 4 > bytes) {
                v &= 0xffffu; // an odd number of uint16 samples
            }
            out[k] = v;
        }
        return;
    }
    if (mode == TSK_CONSTANT) {
        if (threadIdx.x == 0) {
            out[0] = px<F32>(sh, buf, 0);
        }
        return;
    }
    if (seg.n != 0) {
        const uint32_t r = seg.r, b = sh.bits[r], row = sh.row_word[r];
        if (seg.c0 == 0) {
            out[row] = px<F32>(sh, buf, r * w); // seed
            out[row + 1] = b;                   // width word; reserved bytes zero
        }
        if (b != 0) {
            // Residual j (column j + 1) starts at bit j * b of the row's packed words, so the
            // segment's residual k (column c0 + k) starts at bit (c0 + k - 1) * b. The row's first
            // segment thus starts b bits early, in the top of the width word: its residual 0
            // (column 0 against itself) is zero, so every thread appends the same sequence and
            // the width word only has zeros OR-ed into it (after this thread stored it).
            const int32_t start = static_cast<int32_t>(seg.c0 * b) - static_cast<int32_t>(b);
            uint32_t bit = static_cast<uint32_t>(start) & 31u;
            uint32_t at = row + 2 + static_cast<uint32_t>(start >> 5); // row + 1 at column 0
            uint64_t acc = 0;
            // Appends `bits` bits of v (bits <= 32) and flushes a full word.
            auto append = [&](uint32_t v, uint32_t bits) {
                acc |= static_cast<uint64_t>(v) << bit;
                bit += bits;
                if (bit >= 32) {
                    atomicOr(&out[at], static_cast<uint32_t>(acc));
                    acc >>= 32;
                    bit -= 32;
                    ++at;
                }
            };
            if (!F32 && seg.n == kSeg) {
                // uint16 (b <= 16): two residuals joined into one 2b-bit value per append.
                const uint32_t scale = 1u << b;
#pragma unroll
                for (uint32_t k = 0; k < kSeg; k += 2) {
                    append(z[k] + z[k + 1] * scale, 2 * b);
                }
            } else {
#pragma unroll
                for (uint32_t k = 0; k < kSeg; ++k) {
                    if (k < seg.n) {
                        append(z[k], b);
                    }
                }
            }
            if (bit != 0) {
                atomicOr(&out[at], static_cast<uint32_t>(acc));
            }
        }
    }
}

// Index entry of a tile and its payload copied from its slot into the file at `offset` (the
// payload's absolute position), one writer per word.
template <typename Sh>
__device__ void store_tile(const Sh &sh, uint32_t slot, const tsk_encode_image &im,
                           uint64_t index, const TileGeom &g, uint32_t mode, uint32_t length,
                           uint64_t offset) {
    uint8_t *file = reinterpret_cast<uint8_t *>(im.output);
    if (threadIdx.x < 8) {
        uint32_t v = 0;
        switch (threadIdx.x) {
        case 0: v = mode; break;
        case 1: v = g.w | (g.h << 16); break;
        case 2: v = static_cast<uint32_t>(offset); break;
        case 3: v = static_cast<uint32_t>(offset >> 32); break;
        case 4: v = length; break;
        default: v = 0; break;
        }
        put_word(file, 64 + 32 * index + 4 * threadIdx.x, v);
    }
    const uint32_t *in = sh.payload[slot];
    for (uint32_t k = threadIdx.x; k < length / 4; k += kThreads) {
        put_word(file, offset + 4ull * k, in[k]);
    }
}

// The 64-byte header of a finished image (threads 0-15) and its result record.
__device__ void write_header(const tsk_encode_image &im, uint64_t payload_bytes,
                             tsk_result *result) {
    if (threadIdx.x >= 16) {
        return;
    }
    uint8_t *file = reinterpret_cast<uint8_t *>(im.output);
    const uint64_t size = 64 + 32 * im.tile_count + payload_bytes;
    uint32_t v = 0;
    switch (threadIdx.x) {
    case 0: v = 0x00435354u; break; // 'T' 'S' 'C' 0
    case 1: v = 0x0a1a0a0du; break; // 13 10 26 10
    case 2: v = 1u; break;          // version 1.0
    case 3: v = 64u | (im.type << 16); break;
    case 4: v = im.width; break;
    case 5: v = im.height; break;
    case 6: v = im.tile_width | (static_cast<uint32_t>(im.tile_height) << 16); break;
    case 7: v = 32u; break;
    case 8: v = static_cast<uint32_t>(im.tile_count); break;
    case 9: v = static_cast<uint32_t>(im.tile_count >> 32); break;
    case 10: v = 64u; break;
    case 11: v = 0u; break;
    case 12: v = static_cast<uint32_t>(64 + 32 * im.tile_count); break;
    case 13: v = static_cast<uint32_t>((64 + 32 * im.tile_count) >> 32); break;
    case 14: v = static_cast<uint32_t>(size); break;
    default: v = static_cast<uint32_t>(size >> 32); break;
    }
    put_word(file, 4 * threadIdx.x, v);
    if (threadIdx.x == 0) {
        // The launcher cleared the record; a look-back timeout may have set cuda_error.
        result->bytes_written = size;
    }
}

// Sum over the warp of a 64-bit value (every lane gets it).
__device__ __forceinline__ uint64_t warp_sum64(uint64_t v) {
#pragma unroll
    for (uint32_t d = 16; d > 0; d >>= 1) {
        v += __shfl_xor_sync(0xffffffffu, v, d);
    }
    return v;
}

// Images of a batch: a table (plans) or one image passed by value (allocation-free path).
struct ImageTable {
    const tsk_encode_image *images;
    uint32_t count;
    __device__ const tsk_encode_image &operator[](uint32_t i) const {
        return images[i];
    }
    // The image owning batch tile `id`: the last image whose first tile is at or before it.
    __device__ uint32_t owner(uint64_t id) const {
        uint32_t lo = 0, hi = count;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) / 2;
            if (images[mid].first_tile <= id) {
                lo = mid;
            } else {
                hi = mid;
            }
        }
        return lo;
    }
};

struct SingleImage {
    const tsk_encode_image *image;
    __device__ const tsk_encode_image &operator[](uint32_t) const {
        return *image;
    }
    __device__ uint32_t owner(uint64_t) const {
        return 0;
    }
};

// The words whose sum is the lengths published by chunks [stop, g): whole groups inside the
// range from their group words, the chunks before the first whole group and after the last one
// from their own words, numbered 0 .. n-1 in that order (none when stop == g).
struct LookBack {
    const uint64_t *flags, *groups;
    uint64_t stop, lo, head, mid, tail_first, n;
    __device__ LookBack(const uint64_t *f, const uint64_t *gr, uint64_t g, uint64_t s)
        : flags(f), groups(gr), stop(s) {
        lo = (s + kGroupChunks - 1) / kGroupChunks;
        const uint64_t hi = g / kGroupChunks;
        const bool whole = lo < hi;
        head = whole ? lo * kGroupChunks - s : g - s; // chunks from stop
        mid = whole ? hi - lo : 0;                    // groups from lo
        tail_first = whole ? hi * kGroupChunks : g;   // chunks to g
        n = head + mid + (g - tail_first);
    }
    __device__ const uint64_t *word(uint64_t i) const {
        return i < head        ? flags + stop + i
               : i < head + mid ? groups + lo + (i - head)
                                : flags + tail_first + (i - head - mid);
    }
    // The value of word i, given a first load v: reloaded until complete, for a bounded time
    // (then `late` is set and 0 returned).
    __device__ uint64_t value(uint64_t i, uint64_t v, bool &late) const {
        const bool group = i >= head && i < head + mid;
        auto ready = [&](uint64_t w) {
            return group ? (w >> 56) == kGroupChunks : (w >> 62) != 0;
        };
        uint32_t spins = 0;
        while (!ready(v) && spins < (1u << 22)) {
            __nanosleep(64);
            v = ld_relaxed(word(i));
            ++spins;
        }
        if (!ready(v)) {
            late = true;
            return 0;
        }
        return group ? (v & kGroupValue) : (v & kValue);
    }
};

// Sums the lengths published by chunks [stop, g), warp 0 only: each lane loads up to kPerLane of
// every 32 * kPerLane words before it waits on any.
__device__ uint64_t look_back(const uint64_t *flags, const uint64_t *groups, uint64_t g,
                              uint64_t stop, bool &timed_out) {
    constexpr uint32_t kPerLane = 4;
    const uint32_t lane = threadIdx.x % 32;
    const LookBack lb(flags, groups, g, stop);
    uint64_t sum = 0;
    bool late = false;
    for (uint64_t base = 0; base < lb.n; base += 32 * kPerLane) {
        uint64_t v[kPerLane];
#pragma unroll
        for (uint32_t k = 0; k < kPerLane; ++k) {
            const uint64_t i = base + k * 32 + lane;
            v[k] = i < lb.n ? ld_relaxed(lb.word(i)) : 0;
        }
#pragma unroll
        for (uint32_t k = 0; k < kPerLane; ++k) {
            const uint64_t i = base + k * 32 + lane;
            if (i < lb.n) {
                sum += lb.value(i, v[k], late);
            }
        }
    }
    timed_out = __any_sync(0xffffffffu, late);
    return warp_sum64(sum);
}

// The persistent loop. A CTA encodes its chunk c tile by tile; meanwhile it finishes its
// previous chunk c': while c's first tile is analysed, every thread has one word of c''s
// look-back in flight (c' was published a whole chunk earlier, so the chunks before it have
// published theirs), and each later tile of c comes with one tile of c' written out. Then c is
// published and the next chunk, claimed at c's last tile, starts copying in.
template <bool AnyF32, typename Sh, typename Images>
__device__ void encode_chunks(Sh &sh, const Images &images, uint64_t total_tiles,
                              uint32_t chunk_tiles, uint64_t *state, tsk_result *results) {
    uint64_t *counter = state;
    uint64_t *flags = state + 2;
    uint64_t *groups = flags + (total_tiles + chunk_tiles - 1) / chunk_tiles;
    const uint32_t warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    constexpr uint32_t kNone = 3;

    // Thread 0 claims the next chunk into record m.
    auto claim = [&](uint32_t m) {
        const uint64_t g = atomicAdd(reinterpret_cast<unsigned long long *>(counter), 1ull);
        const uint64_t first = g * chunk_tiles;
        Chunk &c = sh.chunks[m];
        c.id = g;
        c.first = first;
        c.count = first < total_tiles ? static_cast<uint32_t>(total_tiles - first < chunk_tiles
                                                                  ? total_tiles - first
                                                                  : chunk_tiles)
                                      : 0u;
    };
    // Thread `t` (t < count) places tile t of claimed chunk m.
    auto place = [&](uint32_t m, uint32_t t) {
        Chunk &c = sh.chunks[m];
        const uint32_t im = images.owner(c.first + t);
        c.image[t] = im;
        c.geom[t] = tile_geom(images[im], c.first + t - images[im].first_tile);
    };
    // Copies tile t of chunk m into buffer `buf` (a cp.async group is closed either way).
    auto prefetch = [&](uint32_t m, uint32_t t, uint32_t buf) {
        const Chunk &c = sh.chunks[m];
        if (t < c.count) {
            issue_tile_any<AnyF32>(sh, buf, images[c.image[t]], c.geom[t]);
        } else {
            cp_async_commit();
        }
    };
    // Warp 0: chunk m's offsets within its images, and the lengths of its last image's tiles
    // published in its own word and added to its group's.
    auto publish = [&](uint32_t m) {
        Chunk &c = sh.chunks[m];
        if (lane == 0) {
            uint64_t run = 0;
            for (uint32_t i = 0; i < c.count; ++i) {
                if (i != 0 && c.image[i] != c.image[i - 1]) {
                    run = 0;
                }
                c.offset[i] = run;
                run += c.length_of[i];
            }
            c.carry = 0;
            c.stop = images[c.image[0]].first_tile / chunk_tiles;
            st_relaxed(flags + c.id, kPublished | run);
            atomicAdd(reinterpret_cast<unsigned long long *>(groups + c.id / kGroupChunks),
                      static_cast<unsigned long long>(kGroupArrival | run));
        }
    };
    // The look-back of chunk m: the chunks of its first image before it (none when the image
    // begins in m).
    auto look_back_of = [&](uint32_t m) {
        const Chunk &c = sh.chunks[m];
        return LookBack(flags, groups, c.id, c.stop);
    };
    // Every thread: word threadIdx.x of chunk m's look-back, loaded early.
    auto early_load = [&](uint32_t m) -> uint64_t {
        const LookBack lb = look_back_of(m);
        return threadIdx.x < lb.n ? ld_relaxed(lb.word(threadIdx.x)) : 0ull;
    };
    // Every thread: its words of chunk m's look-back (the first one given), summed into the
    // chunk's carry; a wait that runs out marks the image's result cuda_error.
    auto settle = [&](uint32_t m, uint64_t early) {
        const LookBack lb = look_back_of(m);
        if (lb.n <= warp * 32) {
            return; // this warp holds none of the words (warp-uniform)
        }
        bool late = false;
        uint64_t sum = 0;
        for (uint64_t i = threadIdx.x; i < lb.n; i += kThreads) {
            sum += lb.value(i, i == threadIdx.x ? early : ld_relaxed(lb.word(i)), late);
        }
        sum = warp_sum64(sum);
        late = __any_sync(0xffffffffu, late);
        if (lane == 0) {
            if (sum != 0) {
                atomicAdd(reinterpret_cast<unsigned long long *>(&sh.chunks[m].carry),
                          static_cast<unsigned long long>(sum));
            }
            if (late) {
                atomicCAS(&results[sh.chunks[m].image[0]].status, 0u, 9u);
            }
        }
    };
    // Tile i of chunk m (its carry complete): index entry and payload; the last tile of an
    // image writes its header.
    auto write_out = [&](uint32_t m, uint32_t i) {
        const Chunk &c = sh.chunks[m];
        const uint32_t im = c.image[i];
        const tsk_encode_image &image = images[im];
        const TileGeom &geom = c.geom[i];
        const uint64_t at = c.offset[i] + (im == c.image[0] ? c.carry : 0);
        store_tile(sh, c.slot0 + i, image, geom.index, geom, c.mode_of[i], c.length_of[i],
                   64 + 32 * image.tile_count + at);
        if (geom.index + 1 == image.tile_count) {
            write_header(image, at + c.length_of[i], results + im);
        }
    };

    uint32_t cur = 0, prev = kNone, next = 1; // chunk records
    if (threadIdx.x == 0) {
        claim(cur);
        sh.chunks[cur].slot0 = 0;
    }
    if (threadIdx.x < TSK_MAX_ROWS) {
        sh.row_or[threadIdx.x] = 0; // then cleared after each tile
    }
    __syncthreads();
    if (sh.chunks[cur].count == 0) {
        return;
    }
    if (threadIdx.x < sh.chunks[cur].count) {
        place(cur, threadIdx.x);
    }
    __syncthreads();
    uint32_t buf = 0; // tile buffer of the next tile to encode
    prefetch(cur, 0, buf);
    for (;;) {
        Chunk &c = sh.chunks[cur];
        const uint32_t count = c.count;
        const uint32_t before = prev != kNone ? sh.chunks[prev].count : 0u; // tiles of c'
        uint64_t early = 0;
        for (uint32_t i = 0; i < count; ++i) {
            const uint32_t slot = c.slot0 + i;
            for (uint32_t k = threadIdx.x; k < sizeof(sh.payload[0]) / 16; k += kThreads) {
                reinterpret_cast<uint4 *>(sh.payload[slot])[k] = make_uint4(0, 0, 0, 0);
            }
            cp_async_wait<0>();
            // Tile i has landed, and every thread is done with the tile before it (its buffer
            // is free).
            __syncthreads();
            if (i + 1 < count) {
                prefetch(cur, i + 1, buf ^ 1);
            } else if (threadIdx.x == 0) {
                claim(next);
            }
            if (i == 0 && before != 0) {
                early = early_load(prev);
            }
            if (i >= 1 && i - 1 < before) {
                write_out(prev, i - 1); // its carry was settled at tile 0
            }
            const tsk_encode_image &im = images[c.image[i]];
            const TileGeom &geom = c.geom[i];
            const Segment seg = segment_of(geom);
            uint32_t z[kSeg];
            if (AnyF32 && im.type == 2) {
                analyze_tile<AnyF32>(sh, buf, geom, seg, z);
                pack_tile<AnyF32>(sh, buf, slot, geom, seg, z);
            } else {
                analyze_tile<false>(sh, buf, geom, seg, z);
                pack_tile<false>(sh, buf, slot, geom, seg, z);
            }
            if (threadIdx.x == 0) {
                c.mode_of[i] = sh.mode;
                c.length_of[i] = sh.length;
            }
            if (threadIdx.x < TSK_MAX_ROWS) {
                sh.row_or[threadIdx.x] = 0; // for the next tile (read before the last barrier)
            }
            if (i == 0 && before != 0) {
                settle(prev, early);
            }
            buf ^= 1;
        }
        __syncthreads();
        // The rest of c' (its carry is complete); then c is published while the next chunk's
        // tiles are placed, and its first tile starts copying in.
        for (uint32_t j = count - 1; j < before; ++j) {
            write_out(prev, j);
        }
        const uint32_t next_count = sh.chunks[next].count;
        if (warp == 0) {
            publish(cur);
        } else if (threadIdx.x - 32 < next_count) {
            place(next, threadIdx.x - 32);
        }
        __syncthreads();
        prefetch(next, 0, buf);
        if (threadIdx.x == 0) {
            sh.chunks[next].slot0 = c.slot0 == 0 ? Sh::kSlots / 2 : 0; // the slots of c'
        }
        const uint32_t spare = prev != kNone ? prev : 2;
        prev = cur;
        cur = next;
        next = spare;
        if (next_count == 0) {
            break;
        }
        __syncthreads();
    }
    // The last chunk: its look-back by warp 0, then its tiles.
    if (warp == 0) {
        const Chunk &c = sh.chunks[prev];
        bool timed_out = false;
        const uint64_t carry = look_back(flags, groups, c.id, c.stop, timed_out);
        if (lane == 0) {
            sh.chunks[prev].carry = carry;
            if (timed_out) {
                atomicCAS(&results[c.image[0]].status, 0u, 9u);
            }
        }
    }
    __syncthreads();
    for (uint32_t j = 0; j < sh.chunks[prev].count; ++j) {
        write_out(prev, j);
    }
}

// AnyF32: the batch has FP32 images (16 KiB tile buffers and payload slots, two slots: one-tile
// chunks, 64 KiB, three CTAs per SM); otherwise 8 KiB buffers and slots, four slots: two-tile
// chunks (48 KiB), four CTAs per SM.
template <bool AnyF32> using SharedFor = EncodeShared<AnyF32 ? 4096u : 2048u, AnyF32 ? 2u : 4u>;
static_assert(SharedFor<false>::kSlots / 2 <= kMaxChunk && SharedFor<true>::kSlots / 2 >= 1,
              "a chunk's tiles fit half the payload slots");

template <bool AnyF32>
__global__ void __launch_bounds__(kThreads, AnyF32 ? 3 : 4)
    encode_kernel(const tsk_encode_image *__restrict__ images, uint32_t image_count,
                  uint64_t total_tiles, uint32_t chunk_tiles, uint64_t *state,
                  tsk_result *results) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    auto &sh = *reinterpret_cast<SharedFor<AnyF32> *>(smem_raw);
    griddep_wait(); // the state and the result records are cleared by encode_clear_kernel
    encode_chunks<AnyF32>(sh, ImageTable{images, image_count}, total_tiles, chunk_tiles, state,
                          results);
}

// Clears a launch's look-back state and its images' result records in one small launch (two
// memsets would be two graph nodes with their own gaps), and lets the encode kernel that
// follows start launching at once: it waits for this grid before it reads either.
__global__ void encode_clear_kernel(uint64_t *state, uint64_t words, tsk_result *results,
                                    uint32_t count) {
    griddep_launch_dependents();
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint64_t first = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    for (uint64_t i = first; i < words; i += stride) {
        state[i] = 0;
    }
    for (uint64_t i = first; i < count; i += stride) {
        results[i] = tsk_result{0, 0, 0};
    }
}

// Tiles per chunk for a launch of `grid` CTAs: as many as spread the tiles over the grid in one
// round, at most half the instance's payload slots (larger batches take several rounds).
uint32_t chunk_tiles_for(uint64_t total_tiles, uint64_t grid, bool any_f32) {
    const uint64_t most = (any_f32 ? SharedFor<true>::kSlots : SharedFor<false>::kSlots) / 2;
    const uint64_t k = (total_tiles + grid - 1) / grid;
    return static_cast<uint32_t>(k < 1 ? 1 : (k > most ? most : k));
}

// Words of state for a launch of `chunks` chunks: the chunk counter, a spare word, one word per
// chunk and one per group of chunks.
uint64_t state_words(uint64_t chunks) {
    return 2 + chunks + (chunks + kGroupChunks - 1) / kGroupChunks;
}

} // namespace
} // namespace tsk

extern "C" uint64_t tsk_encode_state_bytes(uint64_t total_tiles) {
    return 8 * tsk::state_words(total_tiles); // a chunk holds one tile at least
}

extern "C" int tsk_encode_prepare(int device) {
    (void)device;
    // Loads every kernel a compress execution launches (the clear kernel included), so no
    // execution has to.
    cudaFuncAttributes attributes{};
    cudaError_t e = cudaFuncGetAttributes(&attributes, tsk::encode_clear_kernel);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(tsk::encode_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(sizeof(tsk::SharedFor<true>)));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(tsk::encode_kernel<false>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(sizeof(tsk::SharedFor<false>)));
}

extern "C" int tsk_encode_launch(const tsk_encode_image *images, uint32_t image_count,
                                 uint64_t total_tiles, uint32_t any_float, void *state,
                                 tsk_result *results, cudaStream_t stream) {
    if (total_tiles == 0) return cudaSuccess;
    int device = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    auto kernel = any_float ? tsk::encode_kernel<true> : tsk::encode_kernel<false>;
    const size_t smem = any_float ? sizeof(tsk::SharedFor<true>) : sizeof(tsk::SharedFor<false>);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, tsk::kThreads, smem);
    if (e != cudaSuccess) return e;
    uint64_t grid = static_cast<uint64_t>(sms) * (per_sm > 0 ? per_sm : 1);
    const uint32_t k = tsk::chunk_tiles_for(total_tiles, grid, any_float != 0);
    const uint64_t chunks = (total_tiles + k - 1) / k;
    if (grid > chunks) grid = chunks;
    uint64_t *words = static_cast<uint64_t *>(state);
    const uint64_t nwords = tsk::state_words(chunks);
    const uint64_t clear = nwords > image_count ? nwords : image_count;
    const uint32_t clear_grid = static_cast<uint32_t>(clear / 256 + 1 < 1024 ? clear / 256 + 1 : 1024);
    tsk::encode_clear_kernel<<<clear_grid, 256, 0, stream>>>(words, nwords, results, image_count);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // Programmatic dependent launch: the encode grid is scheduled while the clear runs.
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(static_cast<uint32_t>(grid));
    cfg.blockDim = dim3(tsk::kThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, images, image_count, total_tiles, k, words, results);
}

// ---------------------------------------------------------------------------------------------
// Allocation-free encoding of one image.
//
// Some callers cannot allocate device memory when they encode: a process whose GPU memory is
// already reserved in full by another allocator (a framework's caching pool, say), an acquisition
// loop that must not risk an allocator stall or an implicit device synchronization per frame,
// or a deployment that forbids dynamic allocation after initialization. The plan-based
// compress_async path needs device tables from prepare_batch and a caller-allocated workspace;
// this variant needs neither. Its only scratch, the tile counter and look-back flags, lives in
// the file-scope array below, which every GPU that loads the library holds until the process
// exits.
//
// Every call shares that array, and each call clears the part it uses before its kernel runs.
// Two calls that overlap on the same GPU (different streams without an ordering dependency)
// therefore race and corrupt each other's output: order them on one stream or with events.
namespace tsk {
namespace {

// At most kStaticMaxTiles tiles per image. The state is two words, one per chunk and one per 32
// chunks; a chunk holds one tile at least, so 131,070 tiles need at most 2 + 131,070 + 4,096
// words: 1056 KiB.
constexpr uint64_t kStaticMaxTiles = 131070;
constexpr uint64_t kStaticStateWords = 2 + kStaticMaxTiles + (kStaticMaxTiles + 31) / 32;

__device__ __align__(256) uint64_t g_encode_scratch[kStaticStateWords];

template <bool AnyF32>
__global__ void __launch_bounds__(kThreads, AnyF32 ? 3 : 4)
    encode_kernel_static(const __grid_constant__ tsk_encode_image image, uint64_t total_tiles,
                         uint32_t chunk_tiles, uint64_t *state, tsk_result *result) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    auto &sh = *reinterpret_cast<SharedFor<AnyF32> *>(smem_raw);
    encode_chunks<AnyF32>(sh, SingleImage{&image}, total_tiles, chunk_tiles, state, result);
}

// Per-device set-up, done by the first call on each device with that device current: the
// persistent grids of the two instances, from their occupancy. The scratch address and the
// shared-memory attribute are not cached (see static_launch_state), so a device reset between
// calls, which may place the module elsewhere, leaves nothing stale.
struct StaticSetup {
    uint32_t grid[2] = {0, 0}; // persistent grids of the uint16 and FP32 instances
};

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
StaticSetup g_setup[kMaxDevices];

template <bool F32> cudaError_t set_static_smem() {
    return cudaFuncSetAttribute(encode_kernel_static<F32>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(sizeof(SharedFor<F32>)));
}

cudaError_t static_setup(int device, StaticSetup &out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    StaticSetup &s = g_setup[device];
    if (s.grid[0] == 0) {
        int sms = 0;
        cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (e != cudaSuccess) return e;
        for (int f32 = 0; f32 < 2; ++f32) {
            auto kernel = f32 ? encode_kernel_static<true> : encode_kernel_static<false>;
            const size_t smem = f32 ? sizeof(SharedFor<true>) : sizeof(SharedFor<false>);
            e = f32 ? set_static_smem<true>() : set_static_smem<false>();
            if (e != cudaSuccess) return e;
            int per_sm = 0;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, smem);
            if (e != cudaSuccess) return e;
            s.grid[f32] = static_cast<uint32_t>(sms * (per_sm > 0 ? per_sm : 1));
        }
    }
    out = s;
    return cudaSuccess;
}

// What every call looks up afresh (cheap host queries that allocate nothing): the current
// device's address of g_encode_scratch, and the instance's shared-memory limit. In host code
// the name g_encode_scratch is a host-side stand-in, not a device address; the runtime
// returns this device's copy of the array.
cudaError_t static_launch_state(bool f32, uint64_t *&scratch) {
    void *address = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&address, g_encode_scratch);
    if (e != cudaSuccess) return e;
    e = f32 ? set_static_smem<true>() : set_static_smem<false>();
    if (e != cudaSuccess) return e;
    scratch = static_cast<uint64_t *>(address);
    return cudaSuccess;
}

} // namespace
} // namespace tsk

extern "C" uint64_t tsk_encode_static_max_tiles(void) {
    return tsk::kStaticMaxTiles;
}

// Encodes one validated image with the static scratch; allocates nothing. Returns a
// cudaError_t value, or cudaErrorInvalidValue when the image has more tiles than the array holds.
extern "C" int tsk_encode_static_launch(const tsk_encode_image *image, tsk_result *result,
                                        cudaStream_t stream) {
    const uint64_t total = image->tile_count;
    if (total == 0 || total > tsk_encode_static_max_tiles()) return cudaErrorInvalidValue;
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    if (device < 0 || device >= tsk::kMaxDevices) return cudaErrorInvalidDevice;
    tsk::StaticSetup setup;
    e = tsk::static_setup(device, setup);
    if (e != cudaSuccess) return e;
    const bool f32 = image->type == 2;
    uint64_t *scratch = nullptr;
    e = tsk::static_launch_state(f32, scratch);
    if (e != cudaSuccess) return e;
    const uint32_t full = setup.grid[f32 ? 1 : 0];
    const uint32_t k = tsk::chunk_tiles_for(total, full, f32);
    const uint64_t chunks = (total + k - 1) / k;
    const uint64_t grid = full < chunks ? full : chunks;
    const uint64_t words = tsk::state_words(chunks);
    if (words > tsk::kStaticStateWords) return cudaErrorInvalidValue;
    // The array keeps the previous call's contents: clear the counter and this call's words.
    e = cudaMemsetAsync(scratch, 0, 8 * words, stream);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(result, 0, sizeof(tsk_result), stream);
    if (e != cudaSuccess) return e;
    auto kernel = f32 ? tsk::encode_kernel_static<true> : tsk::encode_kernel_static<false>;
    const size_t smem = f32 ? sizeof(tsk::SharedFor<true>) : sizeof(tsk::SharedFor<false>);
    kernel<<<static_cast<uint32_t>(grid), tsk::kThreads, smem, stream>>>(*image, total, k,
                                                                         scratch, result);
    return cudaGetLastError();
}
