// Persistent .tsc tile decoder for sm_100a.
//
// Replaces the reference's one-block-per-tile decode<S,Cal> kernel plus its begin/complete
// kernels (src/cuda/decoder.cu:175-326) with one launch over a flat queue of tile tasks:
//
//  * warp 8 (producer) walks this CTA's tasks and stages each tile's payload into a ring of
//    shared-memory stages: the 16-byte-aligned body with one bulk async copy (TMA engine), the
//    ragged 4-byte head and tail words with cp.async, and the tile's row-start table with a
//    second bulk copy. Completion is an mbarrier transaction count; the consumers release a
//    stage through a second mbarrier. Payload offsets are only 4-byte aligned
//    (docs/format.md:44), so the stage base is shifted by (src & 15) to keep the bulk part
//    aligned on both sides.
//  * warps 0-7 (consumers) decode rows. Each lane owns G consecutive columns: it extracts its
//    residuals from shared-memory words with funnel shifts, undoes the transform (inverse
//    zigzag mod 2^16 for uint16, XOR for FP32 words), scans them in registers, and a segmented
//    warp-shuffle scan over the lanes of the row adds the totals of the groups to its left
//    (decoder.cu:119-173 does the same per row with a lane-sequential group).
//  * RAW and CONSTANT tiles, ROI clipping (prediction still starts at column 0, decoder.cu:247),
//    fused calibration RN(RN(x - offset) * gain) with __fsub_rn/__fmul_rn (device.cuh:81-85),
//    vector stores when a group is aligned, and the trusted encoder-output path (index entry and
//    row walk on the device, decoder.cu:86-110,191-220) all live in the same kernel.
//
// Results: a parsed image cannot fail on the device, so the first task of each image writes its
// DeviceResult directly. Trusted images count finished tasks in the record's reserved field
// (cleared by the planner before the launch); the last one writes the final record, with the
// first failure winning through atomicCAS (decoder.cu:19-22) and the producer's status
// propagated (decoder.cu:314-326).
#include "ptx.cuh"
#include "tasks.h"

#include <cstdint>

namespace tsk {
namespace {

constexpr uint32_t kConsumerWarps = 8;
constexpr uint32_t kConsumers = kConsumerWarps * 32;
constexpr uint32_t kThreads = kConsumers + 32;
constexpr uint32_t kFull = 0xffffffffu;
// A payload stage: the largest tile plus alignment shift and over-read slack.
constexpr uint32_t kStagePayload = TSK_PAYLOAD_BYTES + 128;

enum : uint32_t { kStageOk = 0, kStageSkip = 1, kStageMalformed = 2 };

struct StageHeader {
    tsk_decode_task task;
    uint32_t shift; // byte offset of payload word 0 within the stage buffer
    uint32_t words; // payload words
    uint32_t mode;
    uint32_t state; // kStageOk / kStageSkip / kStageMalformed
};

template <uint32_t Stages> struct Shared {
    alignas(128) uint8_t payload[Stages][kStagePayload];
    alignas(16) uint16_t rows[Stages][TSK_MAX_ROWS];
    alignas(16) StageHeader header[Stages];
    alignas(8) uint64_t full[Stages];
    alignas(8) uint64_t empty[Stages];
    uint32_t valid[Stages]; // trusted row walk verdict of the staged tile
};

// Paths compiled into one kernel instance.
enum : uint32_t { kU16 = 1, kF32 = 2, kPlain = 4, kCal = 8, kTrusted = 16 };

__device__ __forceinline__ uint32_t low_mask(uint32_t bits) {
    return bits >= 32 ? 0xffffffffu : ((1u << bits) - 1u);
}

// Residual term of the inclusive scan (docs/format.md:81-97). uint16: the inverse zigzag as an
// unsigned delta, s = z/2 or -(z/2) - 1, modulo 2^32 (narrowed to 16 bits at the end).
template <bool F32> __device__ __forceinline__ uint32_t term(uint32_t z) {
    if constexpr (F32) {
        return z;
    } else {
        return (z >> 1) ^ (0u - (z & 1u));
    }
}

template <bool F32> __device__ __forceinline__ uint32_t combine(uint32_t a, uint32_t b) {
    if constexpr (F32) {
        return a ^ b;
    } else {
        return a + b;
    }
}

template <bool F32> __device__ __forceinline__ uint32_t uncombine(uint32_t a, uint32_t b) {
    if constexpr (F32) {
        return a ^ b;
    } else {
        return a - b;
    }
}

// Four residuals of at most 16 bits starting at bit pos of the row's packed words: one 64-bit
// window (three shared loads) and funnel shifts, never a shift by 32 (docs/format.md:79).
__device__ __forceinline__ void extract4(const uint32_t *w, uint32_t pos, uint32_t b, uint32_t m,
                                         uint32_t r[4]) {
    const uint32_t q = pos >> 5, s = pos & 31u;
    const uint32_t w0 = w[q], w1 = w[q + 1], w2 = w[q + 2];
    const uint32_t x0 = __funnelshift_r(w0, w1, s);
    const uint32_t x1 = __funnelshift_r(w1, w2, s);
    r[0] = x0 & m;
    r[1] = __funnelshift_rc(x0, x1, b) & m;
    const uint32_t y0 = __funnelshift_rc(x0, x1, 2 * b);
    const uint32_t y1 = __funnelshift_rc(x1, 0u, 2 * b);
    r[2] = y0 & m;
    r[3] = __funnelshift_rc(y0, y1, b) & m;
}

// Two residuals of up to 32 bits starting at bit pos.
__device__ __forceinline__ void extract2(const uint32_t *w, uint32_t pos, uint32_t b, uint32_t m,
                                         uint32_t r[2]) {
    const uint32_t q = pos >> 5, s = pos & 31u;
    const uint32_t w0 = w[q], w1 = w[q + 1], w2 = w[q + 2];
    const uint32_t x0 = __funnelshift_r(w0, w1, s);
    const uint32_t x1 = __funnelshift_r(w1, w2, s);
    r[0] = x0 & m;
    r[1] = __funnelshift_rc(x0, x1, b) & m;
}

// Calibration parameter for output pixel (x, y) (maps are in output-region coordinates).
__device__ __forceinline__ float param(uint64_t map, uint64_t pitch, float scalar, uint64_t x,
                                       uint64_t y) {
    if (map == 0) {
        return scalar;
    }
    return reinterpret_cast<const float *>(map + y * pitch)[x];
}

__device__ __forceinline__ float sample_to_float(uint32_t v, bool f32) {
    return f32 ? __uint_as_float(v) : static_cast<float>(v);
}

// Writes the G decoded values of one lane group: columns [c0, c0 + G) of tile row r.
template <uint32_t G, bool F32, bool Cal>
__device__ __forceinline__ void store_group(const tsk_decode_task &t, const tsk_decode_image &im,
                                            uint32_t r, uint32_t c0, const uint32_t (&v)[G]) {
    const uint32_t col0 = t.col0, col1 = t.col1;
    if (c0 >= col1 || c0 + G <= col0) {
        return;
    }
    const uint64_t oy = static_cast<uint64_t>(t.oy) + (r - t.row0);
    // Output column of tile column c0 (may precede the region when c0 < col0).
    const int64_t ox = static_cast<int64_t>(t.ox) + static_cast<int64_t>(c0) - col0;
    if constexpr (Cal) {
        float f[G];
        const bool whole = c0 >= col0 && c0 + G <= col1;
#pragma unroll
        for (uint32_t k = 0; k < G; ++k) {
            const uint32_t c = c0 + k;
            if (c >= col0 && c < col1) {
                const uint64_t x = static_cast<uint64_t>(ox + k);
                const float value = sample_to_float(v[k], F32);
                f[k] = __fmul_rn(__fsub_rn(value, param(im.offset_map, im.offset_pitch, im.offset,
                                                        x, oy)),
                                 param(im.gain_map, im.gain_pitch, im.gain, x, oy));
            } else {
                f[k] = 0.0f;
            }
        }
        float *line = reinterpret_cast<float *>(im.out + oy * im.out_pitch);
        float *dst = line + ox;
        if (whole && (reinterpret_cast<uintptr_t>(dst) % (4 * G)) == 0) {
            if constexpr (G == 4) {
                *reinterpret_cast<float4 *>(dst) = make_float4(f[0], f[1], f[2], f[3]);
            } else {
                reinterpret_cast<float4 *>(dst)[0] = make_float4(f[0], f[1], f[2], f[3]);
                reinterpret_cast<float4 *>(dst)[1] = make_float4(f[4], f[5], f[6], f[7]);
            }
        } else {
#pragma unroll
            for (uint32_t k = 0; k < G; ++k) {
                const uint32_t c = c0 + k;
                if (c >= col0 && c < col1) {
                    dst[k] = f[k];
                }
            }
        }
    } else if constexpr (F32) {
        uint32_t *dst = reinterpret_cast<uint32_t *>(im.out + oy * im.out_pitch) + ox;
        const bool whole = c0 >= col0 && c0 + G <= col1;
        if (whole && (reinterpret_cast<uintptr_t>(dst) % (4 * G)) == 0) {
            if constexpr (G == 4) {
                *reinterpret_cast<uint4 *>(dst) = make_uint4(v[0], v[1], v[2], v[3]);
            } else {
                reinterpret_cast<uint4 *>(dst)[0] = make_uint4(v[0], v[1], v[2], v[3]);
                reinterpret_cast<uint4 *>(dst)[1] = make_uint4(v[4], v[5], v[6], v[7]);
            }
        } else {
#pragma unroll
            for (uint32_t k = 0; k < G; ++k) {
                const uint32_t c = c0 + k;
                if (c >= col0 && c < col1) {
                    dst[k] = v[k];
                }
            }
        }
    } else {
        uint16_t *dst = reinterpret_cast<uint16_t *>(im.out + oy * im.out_pitch) + ox;
        const bool whole = c0 >= col0 && c0 + G <= col1;
        if (whole && (reinterpret_cast<uintptr_t>(dst) % (2 * G)) == 0) {
            uint32_t p[G / 2];
#pragma unroll
            for (uint32_t k = 0; k < G / 2; ++k) {
                p[k] = (v[2 * k] & 0xffffu) | (v[2 * k + 1] << 16);
            }
            if constexpr (G == 4) {
                *reinterpret_cast<uint2 *>(dst) = make_uint2(p[0], p[1]);
            } else {
                *reinterpret_cast<uint4 *>(dst) = make_uint4(p[0], p[1], p[2], p[3]);
            }
        } else {
#pragma unroll
            for (uint32_t k = 0; k < G; ++k) {
                const uint32_t c = c0 + k;
                if (c >= col0 && c < col1) {
                    dst[k] = static_cast<uint16_t>(v[k]);
                }
            }
        }
    }
}

// Decodes the rows [row0, row1) of one staged tile with the 8 consumer warps.
template <uint32_t G, bool F32, bool Cal>
__device__ void decode_tile(const tsk_decode_task &t, const tsk_decode_image &im,
                            const uint32_t *payload, const uint16_t *rows, uint32_t mode) {
    const uint32_t warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const uint32_t w = t.width;
    // Lanes per row: the smallest power of two whose groups cover the row, at most a warp.
    const uint32_t need = (w + G - 1) / G;
    const uint32_t lw = need >= 32 ? 32 : (need <= 1 ? 1 : 1u << (32 - __clz(need - 1)));
    const uint32_t per_warp = 32 / lw;
    const uint32_t sub = lane & (lw - 1);
    const uint32_t span = G * lw; // columns covered by one pass of a row's lanes
    // Columns 0..col1 must be decoded for prediction; passes beyond col1 are skipped.
    const uint32_t passes = (t.col1 + span - 1) / span;
    const uint32_t first_row = t.row0 + warp * per_warp;
    const uint32_t stride = kConsumerWarps * per_warp;

    for (uint32_t base = first_row; base < t.row1; base += stride) {
        const uint32_t r = base + lane / lw;
        const bool live = r < t.row1;
        if (mode == TSK_PREDICT) {
            const uint32_t *row = payload + (live ? rows[r] : 0u);
            const uint32_t seed = row[0];
            const uint32_t b = row[1] & 0xffu;
            const uint32_t m = low_mask(b);
            const uint32_t *packed = row + 2;
            uint32_t carry = 0;
            for (uint32_t pass = 0; pass < passes; ++pass) {
                const uint32_t c0 = pass * span + sub * G;
                // Residual j belongs to column j + 1; the lane at column 0 starts with the seed.
                const uint32_t j0 = c0 == 0 ? 0u : c0 - 1;
                uint32_t res[G];
                if (live && c0 < w) {
                    if constexpr (F32) {
#pragma unroll
                        for (uint32_t k = 0; k < G; k += 2) {
                            extract2(packed, (j0 + k) * b, b, m, res + k);
                        }
                    } else {
#pragma unroll
                        for (uint32_t k = 0; k < G; k += 4) {
                            extract4(packed, (j0 + k) * b, b, m, res + k);
                        }
                    }
                } else {
#pragma unroll
                    for (uint32_t k = 0; k < G; ++k) {
                        res[k] = 0;
                    }
                }
                uint32_t prefix[G];
                uint32_t total = 0;
#pragma unroll
                for (uint32_t k = 0; k < G; ++k) {
                    const uint32_t c = c0 + k;
                    uint32_t item;
                    if (c0 == 0) {
                        item = k == 0 ? seed : term<F32>(res[k - (k > 0 ? 1 : 0)]);
                    } else {
                        item = term<F32>(res[k]);
                    }
                    item = (live && c < w) ? item : 0u;
                    total = combine<F32>(total, item);
                    prefix[k] = total;
                }
                uint32_t inclusive = total;
                for (uint32_t d = 1; d < lw; d <<= 1) {
                    const uint32_t other = __shfl_up_sync(kFull, inclusive, d, lw);
                    if (sub >= d) {
                        inclusive = combine<F32>(other, inclusive);
                    }
                }
                const uint32_t before = combine<F32>(carry, uncombine<F32>(inclusive, total));
                carry = combine<F32>(carry, __shfl_sync(kFull, inclusive, lw - 1, lw));
                if (live) {
                    uint32_t v[G];
#pragma unroll
                    for (uint32_t k = 0; k < G; ++k) {
                        v[k] = combine<F32>(before, prefix[k]);
                        if constexpr (!F32) {
                            v[k] &= 0xffffu;
                        }
                    }
                    store_group<G, F32, Cal>(t, im, r, c0, v);
                }
            }
        } else if (live) {
            const uint32_t first_pass = t.col0 / span;
            for (uint32_t pass = first_pass; pass < passes; ++pass) {
                const uint32_t c0 = pass * span + sub * G;
                if (c0 >= w) {
                    continue;
                }
                uint32_t v[G];
#pragma unroll
                for (uint32_t k = 0; k < G; ++k) {
                    const uint32_t c = c0 + k;
                    uint32_t value = payload[0];
                    if (mode == TSK_RAW) {
                        const uint32_t index = r * w + (c < w ? c : w - 1);
                        value = F32 ? payload[index] : (payload[index >> 1] >> ((index & 1u) * 16));
                    }
                    v[k] = F32 ? value : (value & 0xffffu);
                }
                store_group<G, F32, Cal>(t, im, r, c0, v);
            }
        }
    }
}

// Reads the row descriptors of an encoder-produced tile (decoder.cu:86-110): false when they do
// not describe exactly the staged payload.
__device__ bool walk_rows(const uint32_t *payload, uint32_t words, uint32_t width,
                          uint32_t height, bool f32, uint16_t *rows) {
    const uint32_t max_bits = f32 ? 32u : 16u;
    uint32_t cursor = 0;
    for (uint32_t r = 0; r < height; ++r) {
        if (words - cursor < 2) {
            return false;
        }
        const uint32_t seed = payload[cursor];
        const uint32_t bits = payload[cursor + 1];
        if (bits > max_bits || (!f32 && seed > 65535u)) {
            return false;
        }
        const uint32_t packed = ((width - 1) * bits + 31) / 32;
        if (words - cursor - 2 < packed) {
            return false;
        }
        rows[r] = static_cast<uint16_t>(cursor);
        cursor += 2 + packed;
    }
    return cursor == words;
}

__device__ __forceinline__ void fail(tsk_result *results, uint32_t image, uint32_t status) {
    atomicCAS(&results[image].status, 0u, status);
}

// Producer: stages task k of this CTA into stage s.
template <uint32_t Stages>
__device__ void stage_task(Shared<Stages> &sh, uint32_t s, const tsk_decode_task &t,
                           const tsk_decode_image *images, const tsk_row_start *rowtab) {
    StageHeader &h = sh.header[s];
    uint64_t src = t.src;
    uint32_t words = static_cast<uint32_t>(t.words_or_tile);
    uint32_t mode = t.mode;
    uint32_t state = kStageOk;
    if (t.flags & TSK_TRUSTED) {
        const tsk_decode_image &im = images[t.image];
        const volatile tsk_result *producer =
            reinterpret_cast<const volatile tsk_result *>(im.encoder_result);
        tsk_result produced;
        produced.status = producer->status;
        produced.bytes_written = producer->bytes_written;
        if (produced.status != 0) {
            state = kStageSkip;
        } else {
            const uint64_t end = produced.bytes_written < im.capacity ? produced.bytes_written
                                                                      : im.capacity;
            const uint8_t *slot = reinterpret_cast<const uint8_t *>(t.src) + 64 +
                                  32 * t.words_or_tile;
            // The archive is only 4-byte aligned: read the entry as 32-bit words.
            const uint32_t *e = reinterpret_cast<const uint32_t *>(slot);
            const uint32_t e0 = e[0], e1 = e[1];
            const uint64_t offset = e[2] | (static_cast<uint64_t>(e[3]) << 32);
            const uint64_t length = e[4] | (static_cast<uint64_t>(e[5]) << 32);
            const uint32_t ew = e1 & 0xffffu, eh = e1 >> 16;
            const uint64_t s_bytes = (t.flags & TSK_F32) ? 4 : 2;
            const uint64_t raw = (static_cast<uint64_t>(t.width) * t.height * s_bytes + 3) / 4 * 4;
            mode = e0 & 0xffu;
            if (mode > TSK_PREDICT || ew != t.width || eh != t.height || offset % 4 != 0 ||
                length % 4 != 0 || length == 0 || length > raw || offset > end ||
                length > end - offset) {
                state = kStageMalformed;
            } else {
                src = t.src + offset;
                words = static_cast<uint32_t>(length / 4);
            }
        }
    }
    const uint32_t shift = static_cast<uint32_t>(src & 15u);
    uint32_t tx = 0;
    if (state == kStageOk) {
        uint8_t *base = sh.payload[s] + shift; // payload word 0
        const uint64_t end = src + 4ull * words;
        const uint64_t a = (src + 15) & ~15ull;
        const uint64_t b = end & ~15ull;
        const uint64_t head_end = a < end ? a : end;
        bool async_words = false;
        for (uint64_t p = src; p < head_end; p += 4) {
            cp_async4(base + (p - src), reinterpret_cast<const void *>(p));
            async_words = true;
        }
        const uint64_t tail_begin = b > a ? b : a;
        for (uint64_t p = tail_begin; p < end; p += 4) {
            cp_async4(base + (p - src), reinterpret_cast<const void *>(p));
            async_words = true;
        }
        if (async_words) {
            cp_async_arrive(&sh.full[s]);
        }
        const uint32_t body = b > a ? static_cast<uint32_t>(b - a) : 0u;
        const bool parsed_rows = !(t.flags & TSK_TRUSTED) && mode == TSK_PREDICT;
        const uint32_t row_bytes = parsed_rows ? (t.height * 2u + 15u) & ~15u : 0u;
        tx = body + row_bytes;
        if (tx != 0) {
            mbar_expect_tx(&sh.full[s], tx);
        }
        if (body != 0) {
            bulk_g2s(base + (a - src), reinterpret_cast<const void *>(a), body, &sh.full[s]);
        }
        if (row_bytes != 0) {
            bulk_g2s(sh.rows[s], rowtab + t.rows_at, row_bytes, &sh.full[s]);
        }
    }
    h.task = t;
    h.shift = shift;
    h.words = words;
    h.mode = mode;
    h.state = state;
    mbar_arrive(&sh.full[s]);
}

template <uint32_t G, uint32_t Stages, uint32_t Paths>
__global__ void __launch_bounds__(kThreads)
    decode_kernel(const tsk_decode_task *__restrict__ tasks, uint32_t ntasks,
                  const tsk_decode_image *__restrict__ images,
                  const tsk_row_start *__restrict__ rowtab, tsk_result *results) {
    extern __shared__ __align__(128) uint8_t smem_raw[];
    Shared<Stages> &sh = *reinterpret_cast<Shared<Stages> *>(smem_raw);
    const uint32_t warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < Stages; ++s) {
            mbar_init(&sh.full[s], 1);
            mbar_init(&sh.empty[s], kConsumerWarps);
        }
        fence_barrier_init();
    }
    __syncthreads();
    const uint32_t mine = blockIdx.x < ntasks ? (ntasks - 1 - blockIdx.x) / gridDim.x + 1 : 0;

    if (warp == kConsumerWarps) {
        // Producer warp: lane 0 issues everything.
        if (lane != 0) {
            return;
        }
        // The next task record is loaded before waiting for a free stage, so its latency
        // overlaps the consumers' work.
        tsk_decode_task t{};
        if (mine != 0) {
            t = tasks[blockIdx.x];
        }
        for (uint32_t i = 0; i < mine; ++i) {
            const uint32_t s = i % Stages;
            tsk_decode_task next{};
            if (i + 1 < mine) {
                next = tasks[blockIdx.x + (i + 1) * gridDim.x];
            }
            if (i >= Stages && !mbar_wait(&sh.empty[s], ((i / Stages) - 1) & 1u)) {
                return; // consumers stopped; they have reported the timeout
            }
            stage_task<Stages>(sh, s, t, images, rowtab);
            t = next;
        }
        return;
    }

    for (uint32_t i = 0; i < mine; ++i) {
        const uint32_t s = i % Stages;
        if (!mbar_wait(&sh.full[s], (i / Stages) & 1u)) {
            if (threadIdx.x == 0) {
                const tsk_decode_task &t = tasks[blockIdx.x + i * gridDim.x];
                fail(results, t.image, 9u); // cuda_error: a staging wait ran out
            }
            return;
        }
        const StageHeader &h = sh.header[s];
        const tsk_decode_task t = h.task;
        const tsk_decode_image &im = images[t.image];
        const uint32_t *payload = reinterpret_cast<const uint32_t *>(sh.payload[s] + h.shift);
        const bool f32 = (t.flags & TSK_F32) != 0;
        const bool cal = (t.flags & TSK_CALIBRATED) != 0;
        bool ok = h.state == kStageOk;
        const uint16_t *rows = sh.rows[s];
        if constexpr ((Paths & kTrusted) != 0) {
            if ((t.flags & TSK_TRUSTED) && ok && h.mode == TSK_PREDICT) {
                if (threadIdx.x == 0) {
                    sh.valid[s] = walk_rows(payload, h.words, t.width, t.height, f32, sh.rows[s]);
                }
                named_sync(1, kConsumers);
                ok = sh.valid[s] != 0;
            }
        }
        if (ok) {
            if constexpr ((Paths & kU16) && (Paths & kPlain)) {
                if (!f32 && !cal) decode_tile<G, false, false>(t, im, payload, rows, h.mode);
            }
            if constexpr ((Paths & kF32) && (Paths & kPlain)) {
                if (f32 && !cal) decode_tile<G, true, false>(t, im, payload, rows, h.mode);
            }
            if constexpr ((Paths & kU16) && (Paths & kCal)) {
                if (!f32 && cal) decode_tile<G, false, true>(t, im, payload, rows, h.mode);
            }
            if constexpr ((Paths & kF32) && (Paths & kCal)) {
                if (f32 && cal) decode_tile<G, true, true>(t, im, payload, rows, h.mode);
            }
        }
        if ((t.flags & TSK_TRUSTED) && threadIdx.x == 0 && h.state == kStageMalformed) {
            fail(results, t.image, 5u); // malformed_data
        }
        if ((t.flags & TSK_TRUSTED) && threadIdx.x == 0 && h.state == kStageOk && !ok) {
            fail(results, t.image, 5u);
        }
        __syncwarp();
        if (lane == 0) {
            mbar_arrive(&sh.empty[s]);
        }
        if (threadIdx.x == 0) {
            if (t.flags & TSK_TRUSTED) {
                // Completion count: the last task of the image writes the final record.
                __threadfence();
                const uint32_t done = atomicAdd(&results[t.image].reserved, 1u);
                if (done + 1 == im.tile_count) {
                    __threadfence();
                    uint32_t status = *reinterpret_cast<volatile uint32_t *>(
                        &results[t.image].status);
                    const uint32_t produced = reinterpret_cast<const volatile tsk_result *>(
                                                  im.encoder_result)
                                                  ->status;
                    if (produced != 0) {
                        status = produced;
                    }
                    results[t.image].reserved = 0;
                    results[t.image].bytes_written = status == 0 ? im.result_bytes : 0;
                    results[t.image].status = status;
                }
            } else if (t.flags & TSK_FIRST) {
                results[t.image].status = 0;
                results[t.image].reserved = 0;
                results[t.image].bytes_written = im.result_bytes;
            }
        }
    }
}

template <uint32_t Stages> constexpr size_t smem_bytes() {
    return sizeof(Shared<Stages>);
}

using KernelFn = void (*)(const tsk_decode_task *, uint32_t, const tsk_decode_image *,
                          const tsk_row_start *, tsk_result *);

constexpr uint32_t kStages = 3;
constexpr uint32_t kAll = kU16 | kF32 | kPlain | kCal | kTrusted;

template <uint32_t G> KernelFn kernel_for() {
    return decode_kernel<G, kStages, kAll>;
}

KernelFn select(uint32_t group) {
    return group == 8 ? kernel_for<8>() : kernel_for<4>();
}

} // namespace
} // namespace tsk

extern "C" int tsk_decode_prepare(tsk_decode_config *config, uint32_t ntasks, int device) {
    const uint32_t group = config->group == 8 ? 8u : 4u;
    auto fn = tsk::select(group);
    const size_t smem = tsk::smem_bytes<tsk::kStages>();
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, tsk::kThreads, smem);
    if (e != cudaSuccess) return e;
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    uint64_t grid = static_cast<uint64_t>(sms) * per_sm;
    if (grid > ntasks) grid = ntasks;
    if (grid < 1) grid = 1;
    config->grid = static_cast<uint32_t>(grid);
    config->group = group;
    config->stages = tsk::kStages;
    return cudaSuccess;
}

extern "C" int tsk_decode_launch(const tsk_decode_task *tasks, uint32_t ntasks,
                                 const tsk_decode_image *images, const tsk_row_start *rows,
                                 tsk_result *results, tsk_decode_config config,
                                 cudaStream_t stream) {
    if (ntasks == 0) return cudaSuccess;
    auto fn = tsk::select(config.group);
    const size_t smem = tsk::smem_bytes<tsk::kStages>();
    fn<<<config.grid, tsk::kThreads, smem, stream>>>(tasks, ntasks, images, rows, results);
    return cudaGetLastError();
}
