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
//  * warps 0-7 (consumers) decode rows. A row is owned by LW lanes (a compile-time width class:
//    the row's columns divided by G); each lane owns G consecutive columns. It loads a 64-bit
//    window of the packed words per group of residuals, extracts them with funnel shifts, undoes
//    the transform (inverse zigzag modulo 2^16 for uint16, XOR for FP32 words) and scans them in
//    registers; an unrolled segmented warp-shuffle scan over the LW lanes adds the totals of the
//    groups to the left, with the row seed as the initial carry (decoder.cu:119-173 does the
//    same per row with a lane-sequential group and a 5-step scan).
//  * RAW and CONSTANT tiles, ROI clipping (prediction still starts at column 0, decoder.cu:247),
//    fused calibration RN(RN(x - offset) * gain) with __fsub_rn/__fmul_rn (device.cuh:81-85),
//    16-byte stores when a group is aligned, and the trusted encoder-output path (index entry and
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
#include <mutex>

namespace tsk {
namespace {

constexpr uint32_t kFull = 0xffffffffu;

// Threads of a CTA with CW consumer warps and, unless the groups stage their own tiles, the
// producer warp.
constexpr uint32_t threads_of(uint32_t cw, bool self = false) {
    return cw * 32 + (self ? 0 : 32);
}

enum : uint32_t { kStageOk = 0, kStageSkip = 1, kStageMalformed = 2, kStageEnd = 3 };

// Everything the consumers need about one staged tile, written by the producer.
struct StageHeader {
    tsk_decode_task task;
    // Calibrated tiles: map addresses of tile column 0 in row row0 (0 for a scalar parameter).
    uint64_t omap, gmap;
    uint64_t opitch, gpitch;
    float offset, gain;
    uint32_t shift; // byte offset of payload word 0 within the stage buffer
    uint32_t words; // payload words
    uint32_t mode;
    uint32_t state; // kStageOk / kStageSkip / kStageMalformed / kStageEnd (no more tasks)
};

// MaxPayload: the largest tile payload of the plan (8 KiB for uint16-only plans, 16 KiB with
// FP32). Each stage adds alignment shift and over-read slack.
//
// Reads stay inside the shared allocation for any payload bytes. A row's residual width comes
// from its descriptor in the payload, clamped to 16 (uint16) or 32 (FP32) bits, and the planner
// keeps every row start inside the payload (check_tile), so a lane's windows end at most
// 8 + 4 * ((width + 28) * bits / 32 + 3) bytes past a row start: 1044 bytes for a 256-wide FP32
// row, 584 for uint16. Metadata built by hand can point a row start anywhere in the payload;
// then the reads of one stage may run into the next stage, and those of the last stage (payload
// end + alignment shift + that reach, less the stage's 128 bytes of slack) into `tail`.
template <uint32_t MaxPayload, uint32_t Stages> struct Shared {
    static constexpr uint32_t kStage = MaxPayload + 128;
    alignas(128) uint8_t payload[Stages][kStage];
    uint8_t tail[MaxPayload > 8192 ? 1152 : 640];
    alignas(16) uint16_t rows[Stages][TSK_MAX_ROWS];
    alignas(16) StageHeader header[Stages];
    alignas(8) uint64_t full[Stages];
    alignas(8) uint64_t empty[Stages];
    uint32_t valid[Stages];   // trusted row walk verdict of the staged tile
    uint32_t rowfail[Stages]; // set when a row check of the group's threads fails
};

// Paths compiled into one kernel instance.
enum : uint32_t { kU16 = 1, kF32 = 2, kPlain = 4, kCal = 8 };

__device__ __forceinline__ uint32_t low_mask(uint32_t bits) {
    return bits >= 32 ? 0xffffffffu : ((1u << bits) - 1u);
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

// Per-task state in registers: output and calibration-map addresses of tile column 0 of the
// first written row (these may lie before the region when the ROI starts inside the tile; they
// are only dereferenced at columns inside it).
struct Ctx {
    uint8_t *out;
    uint64_t pitch;
    const uint8_t *omap;
    uint64_t opitch;
    const uint8_t *gmap;
    uint64_t gpitch;
    float offset, gain;
    uint32_t w, row0, row1, col0, col1;
    bool full;         // TSK_FULL: whole rows of a class width, 16-byte-aligned rows
    uint32_t one, top; // runtime constants 1 and 0x80000000 (see Pipes)
    uint32_t slot;     // this warp's index among the warps that share the tile
};

// Pipe balance. On this SM the integer ALU pipe (logic, shifts, adds) and the FMA pipe
// (integer multiply-add) each run at half the issue rate, and the uint16 decode is ALU-bound.
// Additions written as multiply-adds by a runtime 1 (a kernel argument the compiler cannot
// fold) execute on the FMA pipe instead, and so does the inverse zigzag's sign mask, a high
// product (unzig16).
struct Pipes {
    uint32_t one; // 1
    uint32_t top; // 0x80000000
};

__device__ __forceinline__ uint32_t fma_add(uint32_t a, uint32_t b, const Pipes &p) {
    uint32_t d;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(p.one), "r"(b));
    return d;
}

// Inverse zigzag of the b-bit item whose lowest bit is bit `at` of x, given the rotation
// amount at + 1: the rotation brings the magnitude bits (z >> 1) to bit 0 and the item's low bit
// (the sign of the delta) to bit 31. The sign mask -(z & 1) is then the high word of the signed
// product r * 2 (a multiply-add on the FMA pipe; `two` is 0 for an empty row, whose items are
// all zero), and one logic op masks the magnitude (mh = 2^(b-1) - 1) and applies the sign:
// z/2 or -(z/2) - 1. Exact in the low 16 bits, which is all a uint16 sum uses.
__device__ __forceinline__ uint32_t unzig16(uint32_t x, uint32_t amount, uint32_t mh,
                                            uint32_t two) {
    const uint32_t r = __funnelshift_r(x, x, amount);
    uint32_t sign;
    asm("mul.hi.s32 %0, %1, %2;" : "=r"(sign) : "r"(r), "r"(two));
    return (r & mh) ^ sign;
}

// The 64-bit window of the packed words that starts at the bit of item `first` of a row (item c
// holds residual c - 1; the seed enters as the scan's initial carry). Item 0 starts b bits
// before the packed words, inside the row descriptor's width word, whose bits 8..31 are its
// reserved bytes, zero in every accepted file: for b <= 24 (every uint16 row) item 0 reads as
// zero; wider FP32 rows reach the width byte, so their caller clears item 0.
__device__ __forceinline__ void window(const uint32_t *packed, uint32_t first, uint32_t b,
                                       uint32_t &x0, uint32_t &x1) {
    const int32_t pos = static_cast<int32_t>(first * b) - static_cast<int32_t>(b);
    const int32_t q = pos >> 5; // -1 for item 0
    const uint32_t s = static_cast<uint32_t>(pos) & 31u;
    const uint32_t *w = packed + q;
    const uint32_t w0 = w[0], w1 = w[1], w2 = w[2];
    x0 = __funnelshift_r(w0, w1, s);
    x1 = __funnelshift_r(w1, w2, s);
}

// Keeps only the first nbits bits of the 64-bit window (x1:x0); used for the lanes whose group
// runs past the end of a partial row.
__device__ __forceinline__ void keep_bits(uint32_t &x0, uint32_t &x1, uint32_t nbits) {
    if (nbits < 32) {
        x0 &= (1u << nbits) - 1u;
        x1 = 0;
    } else if (nbits < 64) {
        x1 &= (1u << (nbits - 32)) - 1u;
    }
}

// G scan terms of one lane: columns [c0, c0 + G) of a row of width w with residual width b.
// Partial: the group may run past the end of the row (those items become zero).
template <uint32_t G, bool F32, bool Partial>
__device__ __forceinline__ void terms(const uint32_t *packed, uint32_t c0, uint32_t w, uint32_t b,
                                      const Pipes &pipes, uint32_t (&t)[G]) {
    if constexpr (!F32) {
        // uint16, b <= 16: four residuals per 64-bit window. An empty row (b = 0) has no packed
        // words: its magnitude mask and sign multiplier are zero, so every term is zero whatever
        // the window holds.
        const uint32_t mh = low_mask(b) >> 1;       // the magnitude bits of a zigzag value
        const uint32_t two = b != 0 ? 2u * pipes.one : 0u;
        const uint32_t a1 = b + 1;                  // rotation of the item at bit b
#pragma unroll
        for (uint32_t q = 0; q < G; q += 4) {
            uint32_t x0, x1;
            window(packed, c0 + q, b, x0, x1);
            if constexpr (Partial) {
                if (c0 + q + 4 > w) {
                    const uint32_t items = w > c0 + q ? w - (c0 + q) : 0u;
                    keep_bits(x0, x1, items * b);
                }
            }
            // Items q, q + 1 lie in x0 (2b <= 32 bits) and items q + 2, q + 3 in the word that
            // starts 2b bits later. Inverse zigzag as an unsigned delta: z/2 or -(z/2) - 1.
            const uint32_t y0 = __funnelshift_rc(x0, x1, 2 * b);
            t[q] = unzig16(x0, 1u, mh, two);
            t[q + 1] = unzig16(x0, a1, mh, two);
            t[q + 2] = unzig16(y0, 1u, mh, two);
            t[q + 3] = unzig16(y0, a1, mh, two);
        }
    } else {
        // FP32 words, b <= 32: two residuals per 64-bit window.
        const uint32_t m = low_mask(b);
#pragma unroll
        for (uint32_t q = 0; q < G; q += 2) {
            uint32_t x0, x1;
            window(packed, c0 + q, b, x0, x1);
            if constexpr (Partial) {
                if (c0 + q + 2 > w) {
                    const uint32_t items = w > c0 + q ? w - (c0 + q) : 0u;
                    keep_bits(x0, x1, items * b);
                }
            }
            t[q] = x0 & m;
            t[q + 1] = __funnelshift_rc(x0, x1, b) & m;
        }
        if (c0 == 0) {
            t[0] = 0; // item 0 (see window)
        }
    }
}

__device__ __forceinline__ float cal(float x, float o, float g) {
    return __fmul_rn(__fsub_rn(x, o), g);
}

template <bool F32> __device__ __forceinline__ float as_value(uint32_t v) {
    if constexpr (F32) {
        return __uint_as_float(v);
    } else {
        return static_cast<float>(v & 0xffffu);
    }
}

// Writes the G values of one lane: tile columns [c0, c0 + G) of the row at `line` (address of
// tile column 0). Values are uint16 samples (low halves), FP32 words, or calibrated from them.
// Full: the group is inside the written columns and every address is 16-byte aligned.
template <uint32_t G, bool F32, bool Cal, bool Full>
__device__ __forceinline__ void store(const Ctx &x, uint8_t *line, const uint8_t *orow,
                                      const uint8_t *grow, uint32_t c0, const uint32_t (&v)[G]) {
    if constexpr (!Full) {
        if (c0 >= x.col1 || c0 + G <= x.col0) {
            return;
        }
    }
    bool whole = true;
    if constexpr (!Full) {
        whole = c0 >= x.col0 && c0 + G <= x.col1;
    }
    if constexpr (Cal) {
        float *dst = reinterpret_cast<float *>(line) + c0;
        const float *om = reinterpret_cast<const float *>(orow) + c0;
        const float *gm = reinterpret_cast<const float *>(grow) + c0;
        bool vec = true;
        if constexpr (!Full) {
            vec = whole && ((reinterpret_cast<uintptr_t>(dst) |
                             (orow ? reinterpret_cast<uintptr_t>(om) : 0) |
                             (grow ? reinterpret_cast<uintptr_t>(gm) : 0)) & 15u) == 0;
        }
        if (vec) {
            // Every map load of the group is issued before any store: the output might alias a
            // map as far as the compiler knows, so a load after a store would wait for it.
            float4 o[G / 4], g[G / 4];
#pragma unroll
            for (uint32_t k = 0; k < G; k += 4) {
                o[k / 4] = make_float4(x.offset, x.offset, x.offset, x.offset);
                g[k / 4] = make_float4(x.gain, x.gain, x.gain, x.gain);
                if (orow) o[k / 4] = __ldg(reinterpret_cast<const float4 *>(om + k));
                if (grow) g[k / 4] = __ldg(reinterpret_cast<const float4 *>(gm + k));
            }
#pragma unroll
            for (uint32_t k = 0; k < G; k += 4) {
                const float4 ok = o[k / 4], gk = g[k / 4];
                st_global_v4(dst + k, __float_as_uint(cal(as_value<F32>(v[k]), ok.x, gk.x)),
                             __float_as_uint(cal(as_value<F32>(v[k + 1]), ok.y, gk.y)),
                             __float_as_uint(cal(as_value<F32>(v[k + 2]), ok.z, gk.z)),
                             __float_as_uint(cal(as_value<F32>(v[k + 3]), ok.w, gk.w)));
            }
        } else {
#pragma unroll
            for (uint32_t k = 0; k < G; ++k) {
                const uint32_t c = c0 + k;
                if (c >= x.col0 && c < x.col1) {
                    dst[k] = cal(as_value<F32>(v[k]), orow ? om[k] : x.offset,
                                 grow ? gm[k] : x.gain);
                }
            }
        }
    } else if constexpr (F32) {
        uint32_t *dst = reinterpret_cast<uint32_t *>(line) + c0;
        if (Full || (whole && (reinterpret_cast<uintptr_t>(dst) & 15u) == 0)) {
#pragma unroll
            for (uint32_t k = 0; k < G; k += 4) {
                st_global_v4(dst + k, v[k], v[k + 1], v[k + 2], v[k + 3]);
            }
        } else {
#pragma unroll
            for (uint32_t k = 0; k < G; ++k) {
                const uint32_t c = c0 + k;
                if (c >= x.col0 && c < x.col1) {
                    dst[k] = v[k];
                }
            }
        }
    } else {
        uint16_t *dst = reinterpret_cast<uint16_t *>(line) + c0;
        constexpr uintptr_t kAlign = G >= 8 ? 15u : 2 * G - 1;
        if (Full || (whole && (reinterpret_cast<uintptr_t>(dst) & kAlign) == 0)) {
            uint32_t p[G / 2];
#pragma unroll
            for (uint32_t k = 0; k < G / 2; ++k) {
                p[k] = __byte_perm(v[2 * k], v[2 * k + 1], 0x5410);
            }
            if constexpr (G >= 8) {
#pragma unroll
                for (uint32_t k = 0; k < G / 2; k += 4) {
                    st_global_v4(dst + 2 * k, p[k], p[k + 1], p[k + 2], p[k + 3]);
                }
            } else {
                *reinterpret_cast<uint2 *>(dst) = make_uint2(p[0], p[1]);
            }
        } else {
#pragma unroll
            for (uint32_t k = 0; k < G; ++k) {
                const uint32_t c = c0 + k;
                if (c >= x.col0 && c < x.col1) {
                    dst[k] = static_cast<uint16_t>(v[k]);
                }
            }
        }
    }
}

// a * gate + b on the FMA pipe: with gate 1 (the runtime one) the sum, with gate 0 just b. Used
// where a lane conditionally adds a neighbour's value, so that no branch is needed (the
// compiler cannot predicate an inline-asm statement and would branch around it).
__device__ __forceinline__ uint32_t gated_add(uint32_t a, uint32_t gate, uint32_t b) {
    uint32_t d;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(gate), "r"(b));
    return d;
}

// Decodes rows [row0, row1) of one staged tile with the CW consumer warps; LW lanes per row.
// Full: the tile's width is G * LW (or twice that for FP32 256-wide rows) and every column is
// written to aligned rows, so no per-group bounds or alignment checks are needed.
template <uint32_t CW, uint32_t G, uint32_t LW, bool F32, bool Cal, bool Full>
__device__ void decode_rows(const Ctx &x, const uint32_t *payload, const uint16_t *rows,
                            uint32_t mode) {
    constexpr uint32_t kRowsPerWarp = 32 / LW;
    constexpr uint32_t kSpan = G * LW;
    // CW here: the warps that share the tile; warp: this warp's slot among them.
    const uint32_t warp = CW == 1 ? 0u : x.slot, lane = threadIdx.x % 32;
    const uint32_t sub = lane % LW;
    const uint32_t w = x.w;
    const uint32_t passes = (x.col1 + kSpan - 1) / kSpan;
    const Pipes pipes{x.one, x.top};
    // The scan's combine: XOR for FP32 words, addition (on the FMA pipe) for uint16.
    auto add = [&pipes](uint32_t a, uint32_t b) {
        if constexpr (F32) {
            return a ^ b;
        } else {
            return fma_add(a, b, pipes);
        }
    };
    // Calibration maps are read with plain loads just before each store; their lines are
    // prefetched into L2 a row iteration ahead (and, for a task's first rows, at its start), so
    // those loads do not wait on DRAM. Each address is one this lane reads.
    auto prefetch_maps = [&](uint32_t row) {
        if constexpr (Cal) {
            if (row < x.row1) {
                const uint64_t line = static_cast<uint64_t>(row - x.row0);
                for (uint32_t pass = 0; pass < passes; ++pass) {
                    const uint32_t c0 = pass * kSpan + sub * G;
                    if (c0 < x.col1 && c0 + G > x.col0) {
                        const uint32_t c = c0 > x.col0 ? c0 : x.col0;
                        const uint32_t e = (c0 + G < x.col1 ? c0 + G : x.col1) - 1;
                        if (x.omap) {
                            const uint8_t *m = x.omap + line * x.opitch;
                            asm volatile("prefetch.global.L2 [%0];" ::"l"(m + 4 * c));
                            asm volatile("prefetch.global.L2 [%0];" ::"l"(m + 4 * e));
                        }
                        if (x.gmap) {
                            const uint8_t *m = x.gmap + line * x.gpitch;
                            asm volatile("prefetch.global.L2 [%0];" ::"l"(m + 4 * c));
                            asm volatile("prefetch.global.L2 [%0];" ::"l"(m + 4 * e));
                        }
                    }
                }
            }
        }
    };
    prefetch_maps(x.row0 + warp * kRowsPerWarp + lane / LW);
    for (uint32_t base = x.row0 + warp * kRowsPerWarp; base < x.row1;
         base += CW * kRowsPerWarp) {
        const uint32_t r = base + lane / LW;
        const bool live = r < x.row1;
        prefetch_maps(r + CW * kRowsPerWarp);
        const uint64_t line_off = static_cast<uint64_t>(live ? r - x.row0 : 0u);
        uint8_t *line = x.out + line_off * x.pitch;
        const uint8_t *orow = nullptr, *grow = nullptr;
        if constexpr (Cal) {
            orow = x.omap ? x.omap + line_off * x.opitch : nullptr;
            grow = x.gmap ? x.gmap + line_off * x.gpitch : nullptr;
        }
        if (mode == TSK_PREDICT) {
            const uint32_t *row = payload + (live ? rows[r] : 0u);
            const uint32_t width_byte = live ? (row[1] & 0xffu) : 0u;
            const uint32_t b = width_byte < (F32 ? 32u : 16u) ? width_byte : (F32 ? 32u : 16u);
            const uint32_t *packed = row + 2;
            // The seed is the initial carry: value(c) = seed (+ or ^) the terms of items 0..c.
            uint32_t carry = live ? row[0] : 0u;
            for (uint32_t pass = 0; pass < passes; ++pass) {
                const uint32_t c0 = pass * kSpan + sub * G;
                uint32_t t[G];
                if (Full || c0 < w) {
                    terms<G, F32, !Full>(packed, c0, w, b, pipes, t);
                } else {
#pragma unroll
                    for (uint32_t k = 0; k < G; ++k) {
                        t[k] = 0;
                    }
                }
                // Two independent running sums over the halves of the group (half the
                // dependency chain), joined when the outputs are formed.
                constexpr uint32_t H = G / 2;
#pragma unroll
                for (uint32_t k = 1; k < G; ++k) {
                    if (k != H) {
                        t[k] = add(t[k - 1], t[k]);
                    }
                }
                const uint32_t total = add(t[H - 1], t[G - 1]);
                uint32_t inclusive = total;
#pragma unroll
                for (uint32_t d = 1; d < LW; d <<= 1) {
                    const uint32_t other = __shfl_up_sync(kFull, inclusive, d, LW);
                    // Branch-free conditional add (see gated_add).
                    if constexpr (F32) {
                        inclusive ^= sub >= d ? other : 0u;
                    } else {
                        inclusive = gated_add(other, sub >= d ? x.one : 0u, inclusive);
                    }
                }
                const uint32_t before = add(carry, uncombine<F32>(inclusive, total));
                carry = add(carry, __shfl_sync(kFull, inclusive, LW - 1, LW));
                if (live) {
                    const uint32_t mid = add(before, t[H - 1]);
                    uint32_t v[G];
#pragma unroll
                    for (uint32_t k = 0; k < G; ++k) {
                        v[k] = add(k < H ? before : mid, t[k]);
                    }
                    store<G, F32, Cal, Full>(x, line, orow, grow, c0, v);
                }
            }
        } else if (live) {
            for (uint32_t pass = x.col0 / kSpan; pass < passes; ++pass) {
                const uint32_t c0 = pass * kSpan + sub * G;
                if (!Full && c0 >= w) {
                    continue;
                }
                uint32_t v[G];
#pragma unroll
                for (uint32_t k = 0; k < G; ++k) {
                    const uint32_t c = Full || c0 + k < w ? c0 + k : w - 1;
                    if (mode == TSK_RAW) {
                        const uint32_t index = r * w + c;
                        v[k] = F32 ? payload[index]
                                   : reinterpret_cast<const uint16_t *>(payload)[index];
                    } else {
                        v[k] = F32 ? payload[0] : (payload[0] & 0xffffu);
                    }
                }
                store<G, F32, Cal, Full>(x, line, orow, grow, c0, v);
            }
        }
    }
}

// Predictive uint16 rows. The class width G * LW covers every uint16 row (64, 128 or 256), so
// a row is one pass of its LW lanes: no pass loop and no carry between passes. Each lane
// decodes NR rows at once (rows r, r + R, ... with R = CW * 32 / LW), their steps interleaved so
// that one row's shuffle scan and window loads overlap the other rows' arithmetic. The inner
// loop has no branches: the scan's conditional adds are gated multiply-adds, and AllLive (every
// row of every iteration exists: the common whole-tile case) drops the per-row checks.
template <uint32_t CW, uint32_t G, uint32_t LW, bool Cal, bool Full, uint32_t NR, bool AllLive>
__device__ __forceinline__ void predict_rows_u16(const Ctx &x, const uint32_t *payload,
                                                 const uint16_t *rows) {
    constexpr uint32_t kRowsPerWarp = 32 / LW;
    constexpr uint32_t kStride = CW * kRowsPerWarp;
    constexpr uint32_t H = G / 2;
    constexpr uint32_t kSteps = LW == 1 ? 0 : LW == 2 ? 1 : LW == 4 ? 2 : LW == 8 ? 3 : LW == 16 ? 4 : 5;
    // CW here: the warps that share the tile; warp: this warp's slot among them.
    const uint32_t warp = CW == 1 ? 0u : x.slot, lane = threadIdx.x % 32;
    const uint32_t sub = lane % LW;
    const uint32_t c0 = sub * G;
    const uint32_t w = x.w;
    const Pipes pipes{x.one, x.top};
    auto add = [&pipes](uint32_t a, uint32_t b) { return fma_add(a, b, pipes); };
    // gate[j]: 1 when this lane takes the value 2^j lanes to its left in scan step j.
    uint32_t gate[kSteps > 0 ? kSteps : 1];
#pragma unroll
    for (uint32_t j = 0; j < kSteps; ++j) {
        gate[j] = sub >= (1u << j) ? x.one : 0u;
    }
    auto prefetch_maps = [&](uint32_t row) {
        if constexpr (Cal) {
            if (row < x.row1 && c0 < x.col1 && c0 + G > x.col0) {
                const uint64_t line = static_cast<uint64_t>(row - x.row0);
                const uint32_t c = c0 > x.col0 ? c0 : x.col0;
                const uint32_t e = (c0 + G < x.col1 ? c0 + G : x.col1) - 1;
                if (x.omap) {
                    const uint8_t *m = x.omap + line * x.opitch;
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(m + 4 * c));
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(m + 4 * e));
                }
                if (x.gmap) {
                    const uint8_t *m = x.gmap + line * x.gpitch;
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(m + 4 * c));
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(m + 4 * e));
                }
            }
        }
    };
    const uint32_t mine = x.row0 + warp * kRowsPerWarp + lane / LW;
    if constexpr (Cal) {
#pragma unroll
        for (uint32_t n = 0; n < NR; ++n) {
            prefetch_maps(mine + n * kStride);
        }
    }
    for (uint32_t base = x.row0 + warp * kRowsPerWarp; base < x.row1; base += NR * kStride) {
        uint32_t t[NR][G];
        uint32_t carry[NR], total[NR], inclusive[NR];
        bool live[NR];
        uint64_t line_off[NR];
#pragma unroll
        for (uint32_t n = 0; n < NR; ++n) {
            const uint32_t r = base + n * kStride + lane / LW;
            live[n] = AllLive || r < x.row1;
            if constexpr (Cal) {
                prefetch_maps(r + NR * kStride);
            }
            line_off[n] = static_cast<uint64_t>(live[n] ? r - x.row0 : 0u);
            const uint32_t *row = payload + (live[n] ? rows[r] : 0u);
            const uint32_t width_byte = row[1] & 0xffu;
            const uint32_t b = width_byte < 16u ? width_byte : 16u;
            carry[n] = row[0];
            if (Full || c0 < w) {
                terms<G, false, !Full>(row + 2, c0, w, b, pipes, t[n]);
            } else {
#pragma unroll
                for (uint32_t k = 0; k < G; ++k) {
                    t[n][k] = 0;
                }
            }
        }
#pragma unroll
        for (uint32_t n = 0; n < NR; ++n) {
#pragma unroll
            for (uint32_t k = 1; k < G; ++k) {
                if (k != H) {
                    t[n][k] = add(t[n][k - 1], t[n][k]);
                }
            }
            total[n] = add(t[n][H - 1], t[n][G - 1]);
            inclusive[n] = total[n];
        }
#pragma unroll
        for (uint32_t j = 0; j < kSteps; ++j) {
#pragma unroll
            for (uint32_t n = 0; n < NR; ++n) {
                const uint32_t other = __shfl_up_sync(kFull, inclusive[n], 1u << j, LW);
                inclusive[n] = gated_add(other, gate[j], inclusive[n]);
            }
        }
#pragma unroll
        for (uint32_t n = 0; n < NR; ++n) {
            if (AllLive || live[n]) {
                const uint32_t before = add(carry[n], inclusive[n] - total[n]);
                const uint32_t mid = add(before, t[n][H - 1]);
                uint32_t v[G];
#pragma unroll
                for (uint32_t k = 0; k < G; ++k) {
                    v[k] = add(k < H ? before : mid, t[n][k]);
                }
                uint8_t *line = x.out + line_off[n] * x.pitch;
                const uint8_t *orow = nullptr, *grow = nullptr;
                if constexpr (Cal) {
                    orow = x.omap ? x.omap + line_off[n] * x.opitch : nullptr;
                    grow = x.gmap ? x.gmap + line_off[n] * x.gpitch : nullptr;
                }
                store<G, false, Cal, Full>(x, line, orow, grow, c0, v);
            }
        }
    }
}

// Predictive FP32 rows: the same single-pass structure as predict_rows_u16 with G columns per
// lane (G * LW is the class width: 64, 128 or 256 FP32 words, so a row is one pass), residuals
// undone with XOR. The running XOR and the scan's conditional XOR need no multiply: a lane
// takes its left neighbour's total masked by an all-ones or zero gate.
template <uint32_t CW, uint32_t G, uint32_t LW, bool Cal, bool Full, bool AllLive>
__device__ __forceinline__ void predict_rows_f32(const Ctx &x, const uint32_t *payload,
                                                 const uint16_t *rows) {
    constexpr uint32_t kRowsPerWarp = 32 / LW;
    constexpr uint32_t kStride = CW * kRowsPerWarp;
    constexpr uint32_t H = G / 2;
    constexpr uint32_t kSteps = LW == 1 ? 0 : LW == 2 ? 1 : LW == 4 ? 2 : LW == 8 ? 3 : LW == 16 ? 4 : 5;
    // CW here: the warps that share the tile; warp: this warp's slot among them.
    const uint32_t warp = CW == 1 ? 0u : x.slot, lane = threadIdx.x % 32;
    const uint32_t sub = lane % LW;
    const uint32_t c0 = sub * G;
    const uint32_t w = x.w;
    const Pipes pipes{x.one, x.top};
    uint32_t gate[kSteps > 0 ? kSteps : 1];
#pragma unroll
    for (uint32_t j = 0; j < kSteps; ++j) {
        gate[j] = sub >= (1u << j) ? 0xffffffffu : 0u;
    }
    auto prefetch_maps = [&](uint32_t row) {
        if constexpr (Cal) {
            if (row < x.row1 && c0 < x.col1 && c0 + G > x.col0) {
                const uint64_t line = static_cast<uint64_t>(row - x.row0);
                const uint32_t c = c0 > x.col0 ? c0 : x.col0;
                const uint32_t e = (c0 + G < x.col1 ? c0 + G : x.col1) - 1;
                if (x.omap) {
                    const uint8_t *m = x.omap + line * x.opitch;
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(m + 4 * c));
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(m + 4 * e));
                }
                if (x.gmap) {
                    const uint8_t *m = x.gmap + line * x.gpitch;
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(m + 4 * c));
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(m + 4 * e));
                }
            }
        }
    };
    if constexpr (Cal) {
        prefetch_maps(x.row0 + warp * kRowsPerWarp + lane / LW);
    }
    for (uint32_t base = x.row0 + warp * kRowsPerWarp; base < x.row1; base += kStride) {
        const uint32_t r = base + lane / LW;
        const bool live = AllLive || r < x.row1;
        if constexpr (Cal) {
            prefetch_maps(r + kStride);
        }
        const uint64_t line_off = static_cast<uint64_t>(live ? r - x.row0 : 0u);
        const uint32_t *row = payload + (live ? rows[r] : 0u);
        const uint32_t width_byte = row[1] & 0xffu;
        const uint32_t b = width_byte < 32u ? width_byte : 32u;
        const uint32_t carry = row[0];
        uint32_t t[G];
        if (Full || c0 < w) {
            terms<G, true, !Full>(row + 2, c0, w, b, pipes, t);
        } else {
#pragma unroll
            for (uint32_t k = 0; k < G; ++k) {
                t[k] = 0;
            }
        }
#pragma unroll
        for (uint32_t k = 1; k < G; ++k) {
            if (k != H) {
                t[k] ^= t[k - 1];
            }
        }
        const uint32_t total = t[H - 1] ^ t[G - 1];
        uint32_t inclusive = total;
#pragma unroll
        for (uint32_t j = 0; j < kSteps; ++j) {
            const uint32_t other = __shfl_up_sync(kFull, inclusive, 1u << j, LW);
            inclusive ^= other & gate[j];
        }
        if (AllLive || live) {
            const uint32_t before = carry ^ inclusive ^ total;
            const uint32_t mid = before ^ t[H - 1];
            uint32_t v[G];
#pragma unroll
            for (uint32_t k = 0; k < G; ++k) {
                v[k] = (k < H ? before : mid) ^ t[k];
            }
            uint8_t *line = x.out + line_off * x.pitch;
            const uint8_t *orow = nullptr, *grow = nullptr;
            if constexpr (Cal) {
                orow = x.omap ? x.omap + line_off * x.opitch : nullptr;
                grow = x.gmap ? x.gmap + line_off * x.gpitch : nullptr;
            }
            store<G, true, Cal, Full>(x, line, orow, grow, c0, v);
        }
    }
}

template <uint32_t CW, uint32_t G, uint32_t LW, bool F32, bool Cal, uint32_t NR>
__device__ __forceinline__ void decode_class(const Ctx &x, const uint32_t *payload,
                                             const uint16_t *rows, uint32_t mode) {
    if constexpr (F32 && NR != 0) {
        if (mode == TSK_PREDICT) {
            constexpr uint32_t kRowsPerIteration = CW * (32 / LW);
            if (x.full && (x.row1 - x.row0) % kRowsPerIteration == 0) {
                predict_rows_f32<CW, G, LW, Cal, true, true>(x, payload, rows);
            } else if (x.full) {
                predict_rows_f32<CW, G, LW, Cal, true, false>(x, payload, rows);
            } else {
                predict_rows_f32<CW, G, LW, Cal, false, false>(x, payload, rows);
            }
            return;
        }
    }
    if constexpr (!F32 && NR != 0) {
        if (mode == TSK_PREDICT) {
            constexpr uint32_t kRowsPerIteration = NR * CW * (32 / LW);
            if (x.full && (x.row1 - x.row0) % kRowsPerIteration == 0) {
                predict_rows_u16<CW, G, LW, Cal, true, NR, true>(x, payload, rows);
            } else if (x.full) {
                predict_rows_u16<CW, G, LW, Cal, true, NR, false>(x, payload, rows);
            } else {
                predict_rows_u16<CW, G, LW, Cal, false, NR, false>(x, payload, rows);
            }
            return;
        }
    }
    if (x.full) {
        decode_rows<CW, G, LW, F32, Cal, true>(x, payload, rows, mode);
    } else {
        decode_rows<CW, G, LW, F32, Cal, false>(x, payload, rows, mode);
    }
}

// Width classes: a row of the class width is covered by LW = width / G lanes. uint16 rows take
// G16 columns per lane (8 or 16), FP32 rows 4.
// NR: uint16 predictive rows decoded per lane at once by predict_rows_u16 (0 keeps them on
// the generic decode_rows).
template <uint32_t CW, uint32_t G16, bool F32, bool Cal, uint32_t NR>
__device__ __forceinline__ void decode_tile(const Ctx &x, const uint32_t *payload,
                                            const uint16_t *rows, uint32_t mode) {
    if constexpr (!F32) {
        if (x.w > 128) {
            decode_class<CW, G16, 256 / G16, false, Cal, NR>(x, payload, rows, mode);
        } else if (x.w > 64) {
            decode_class<CW, G16, 128 / G16, false, Cal, NR>(x, payload, rows, mode);
        } else {
            decode_class<CW, G16, 64 / G16, false, Cal, NR>(x, payload, rows, mode);
        }
    } else if constexpr (NR != 0) {
        // 16 FP32 words per lane: every class width is one pass.
        if (x.w > 128) {
            decode_class<CW, 16, 16, true, Cal, NR>(x, payload, rows, mode);
        } else if (x.w > 64) {
            decode_class<CW, 16, 8, true, Cal, NR>(x, payload, rows, mode);
        } else {
            decode_class<CW, 16, 4, true, Cal, NR>(x, payload, rows, mode);
        }
    } else {
        if (x.w > 64) {
            decode_class<CW, 4, 32, true, Cal, 0>(x, payload, rows, mode);
        } else {
            decode_class<CW, 4, 16, true, Cal, 0>(x, payload, rows, mode);
        }
    }
}

// Locates the row descriptors of a tile whose rows are read on the device (encoder output,
// reference decoder.cu:86-110, and unparsed files): the serial part of the row walk, one lane.
// Each row starts where the previous one's packed words end; a width word above the widest
// sample (which also catches nonzero reserved bytes, as the word is compared whole) or a row
// that does not fit ends the walk. False unless the rows end exactly at the payload's end.
// The per-row checks that need no chain run on every thread of the group (row_ok).
//
// The loop carries as little as it can: the width word of a row that starts past the payload's
// end is read from the stage's slack (the stage holds a whole tile plus slack, and the walk
// stops as soon as a row ends past the payload, so it reads at most one word beyond it), and
// the row is then rejected by the end check, which covers the descriptor's own two words.
__device__ bool chain_rows(const uint32_t *payload, uint32_t words, uint32_t width,
                           uint32_t height, bool f32, uint16_t *rows) {
    const uint32_t max_bits = f32 ? 32u : 16u, wm1 = width - 1;
    uint32_t cursor = 0;
    for (uint32_t r = 0; r < height; ++r) {
        const uint32_t bits = payload[cursor + 1];
        rows[r] = static_cast<uint16_t>(cursor);
        cursor += 2 + ((wm1 * (bits <= max_bits ? bits : 0u) + 31) >> 5);
        if (bits > max_bits || cursor > words) {
            return false;
        }
    }
    return cursor == words;
}

// The checks of one located row: the seed of a uint16 row is a uint16 value; strict (unparsed
// files) adds the host parser's remaining row rules (parser.cpp check_payloads, after reference
// src/cpu/parser.cpp:127-171): a one-column tile has zero-width rows, and the unused high bits
// of the row's last packed word are zero.
__device__ __forceinline__ bool row_ok(const uint32_t *payload, uint32_t start, uint32_t width,
                                       bool f32, bool strict) {
    const uint32_t seed = payload[start], bits = payload[start + 1];
    if (!f32 && seed > 65535u) {
        return false;
    }
    if (strict) {
        const uint32_t nbits = (width - 1) * bits, packed = (nbits + 31) / 32;
        if ((width == 1 && bits != 0) ||
            (nbits % 32 != 0 && (payload[start + 1 + packed] >> (nbits % 32)) != 0)) {
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ void fail(tsk_result *results, uint32_t image, uint32_t status) {
    atomicCAS(&results[image].status, 0u, status);
}

// A 64-byte task record through the read-only path (records are never written during a launch).
__device__ __forceinline__ tsk_decode_task load_task(const tsk_decode_task *p) {
    union {
        uint4 v[4];
        tsk_decode_task t;
    } u;
    for (int k = 0; k < 4; ++k) {
        u.v[k] = ld_nc_v4(reinterpret_cast<const uint4 *>(p) + k);
    }
    return u.t;
}

// Task sources of the persistent loop. The producer asks a source for the task at queue index
// g = blockIdx.x + i * gridDim.x (increasing i); the consumers ask it for the calibration and
// the bytes_written of a task's image.
//
// TableSource: a planned queue of tasks and its image table (every plan and mixed batch).
struct TableSource {
    static constexpr bool kTrusted = true;
    static constexpr bool kLocalCounts = false;
    const tsk_decode_task *tasks;
    const tsk_decode_image *images;
    uint32_t ntasks;
    uint32_t *claims; // the device work queue's counter (dynamic instances), else unused

    __device__ tsk_decode_task task(uint32_t g) {
        return load_task(tasks + g);
    }
    __device__ uint32_t image_of(uint32_t g) const {
        return tasks[g].image;
    }
    __device__ const tsk_decode_image &image(uint32_t i) const {
        return images[i];
    }
    __device__ void calibration(const tsk_decode_task &t, StageHeader &h) const {
        const tsk_decode_image &im = images[t.image];
        const int64_t cx = static_cast<int64_t>(t.ox) - t.col0;
        h.offset = im.offset;
        h.gain = im.gain;
        h.opitch = im.offset_pitch;
        h.gpitch = im.gain_pitch;
        h.omap = im.offset_map ? im.offset_map + t.oy * im.offset_pitch + cx * 4 : 0;
        h.gmap = im.gain_map ? im.gain_map + t.oy * im.gain_pitch + cx * 4 : 0;
    }
    __device__ uint64_t result_bytes(const tsk_decode_task &t) const {
        return images[t.image].result_bytes;
    }
};

// ServeSource: a serving batch (the kernel's parameter block) over resident archives. Task g
// is tile l = g - (first task of its request) of the request's ROI in row-major tile order;
// its template is completed with the ROI clip that the host planner applies per task
// (plan.cpp clip(), after reference plan.cpp:281-349), so no task table is uploaded.
struct ServeSource {
    static constexpr bool kTrusted = false;
    static constexpr bool kLocalCounts = false;
    const tsk_serve_batch *batch;
    const tsk_serve_archive *archives;
    uint32_t ntasks;
    uint32_t cursor; // request of the last task asked for (indexes only increase)

    __device__ tsk_decode_task task(uint32_t g) {
        const tsk_serve_request *req = batch->requests;
        while (g >= req[cursor].task_end) {
            ++cursor; // g < ntasks == req[count - 1].task_end ends the walk
        }
        const tsk_serve_request &q = req[cursor];
        const uint32_t l = g - (cursor != 0 ? req[cursor - 1].task_end : 0u);
        const tsk_serve_archive &a = archives[q.archive];
        const uint32_t trow = q.top + l / q.across;
        const uint32_t tcol = q.left + l % q.across;
        const tsk_decode_task *tpl = reinterpret_cast<const tsk_decode_task *>(a.tiles) +
                                     static_cast<uint64_t>(trow) * a.tiles_across + tcol;
        tsk_decode_task t = load_task(tpl);
        t.image = cursor;
        t.flags = static_cast<uint8_t>(t.flags | q.flags | (l == 0 ? TSK_FIRST : 0));
        const uint64_t x = static_cast<uint64_t>(tcol) * a.tile_width;
        const uint64_t y = static_cast<uint64_t>(trow) * a.tile_height;
        const uint64_t rx1 = static_cast<uint64_t>(q.x) + q.width;
        const uint64_t ry1 = static_cast<uint64_t>(q.y) + q.height;
        t.row0 = static_cast<uint16_t>(q.y > y ? q.y - y : 0);
        t.row1 = static_cast<uint16_t>(ry1 < y + t.height ? ry1 - y : t.height);
        t.col0 = static_cast<uint16_t>(q.x > x ? q.x - x : 0);
        t.col1 = static_cast<uint16_t>(rx1 < x + t.width ? rx1 - x : t.width);
        t.ox = static_cast<uint32_t>(x + t.col0 - q.x);
        t.oy = static_cast<uint32_t>(y + t.row0 - q.y);
        const uint64_t esize = (t.flags & (TSK_F32 | TSK_CALIBRATED)) ? 4 : 2;
        // Unsigned wrap-around gives the address before the region when t.ox < t.col0.
        t.dst = q.out + t.oy * q.out_pitch + (static_cast<uint64_t>(t.ox) - t.col0) * esize;
        t.pitch = q.out_pitch;
        const bool class_width = t.width == 64 || t.width == 128 || t.width == 256;
        if (class_width && t.col0 == 0 && t.col1 == t.width && ((t.dst | t.pitch) & 15u) == 0) {
            t.flags |= TSK_FULL;
        }
        return t;
    }
    __device__ uint32_t image_of(uint32_t g) const {
        uint32_t r = 0;
        while (r + 1 < batch->count && g >= batch->requests[r].task_end) {
            ++r;
        }
        return r;
    }
    __device__ const tsk_decode_image &image(uint32_t) const; // no trusted tasks
    __device__ void calibration(const tsk_decode_task &t, StageHeader &h) const {
        const tsk_serve_request &q = batch->requests[t.image];
        h.offset = q.offset;
        h.gain = q.gain;
        h.opitch = h.gpitch = 0;
        h.omap = h.gmap = 0;
    }
    __device__ uint64_t result_bytes(const tsk_decode_task &t) const {
        const tsk_serve_request &q = batch->requests[t.image];
        const uint64_t esize = (t.flags & (TSK_F32 | TSK_CALIBRATED)) ? 4 : 2;
        return static_cast<uint64_t>(q.width) * q.height * esize;
    }
};

// FileSource: unparsed .tsc files (the kernel's parameter block), each decoded whole. Task g is
// tile l = g - (first task of its file) of its file, in index order. Its index entry and rows
// are read and validated on the device (TSK_TRUSTED | TSK_UNPARSED), so nothing but the file
// records is passed. The first task of a file also compares the file's 64 header bytes with
// the copy the host checked; a difference marks the task (reserved = 1), and staging reports
// it as malformed data.
struct FileSource {
    static constexpr bool kTrusted = true;
    static constexpr bool kLocalCounts = true;
    const tsk_file_batch *batch;
    uint32_t ntasks;
    uint32_t cursor; // file of the last task asked for (indexes only increase)
    uint32_t *done;  // shared memory: this CTA's finished tiles per file

    // Adds this CTA's finished tiles of file k to its record's count; the CTA that completes
    // the count writes the final record (the failures CAS-ed before are visible to it).
    __device__ void flush(uint32_t k, tsk_result *results) const {
        const uint32_t c = done[k];
        if (c == 0) {
            return;
        }
        const tsk_decode_image &im = batch->files[k].image;
        __threadfence();
        const uint32_t before = atomicAdd(&results[k].reserved, c);
        if (before + c == im.tile_count) {
            __threadfence();
            const uint32_t status = *reinterpret_cast<volatile uint32_t *>(&results[k].status);
            results[k].reserved = 0;
            results[k].bytes_written = status == 0 ? im.result_bytes : 0;
            results[k].status = status;
        }
    }

    __device__ tsk_decode_task task(uint32_t g) {
        const tsk_file *files = batch->files;
        while (g >= files[cursor].task_end) {
            ++cursor; // g < ntasks == files[count - 1].task_end ends the walk
        }
        const tsk_file &f = files[cursor];
        const tsk_decode_image &im = f.image;
        const uint32_t l = g - (cursor != 0 ? files[cursor - 1].task_end : 0u);
        const uint32_t trow = l / f.tiles_across, tcol = l % f.tiles_across;
        const uint64_t x = static_cast<uint64_t>(tcol) * im.tile_width;
        const uint64_t y = static_cast<uint64_t>(trow) * im.tile_height;
        // The producer asks for a task one tile ahead: its index entry (and the previous one,
        // for the payload chain) is on its way to L2 when the tile is staged.
        asm volatile("prefetch.global.L2 [%0];" ::"l"(f.src + 32 + 32ull * l));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(f.src + 64 + 32ull * l));
        tsk_decode_task t{};
        t.src = f.src;
        t.words_or_tile = l;
        t.image = cursor;
        t.width = static_cast<uint16_t>(min(static_cast<uint64_t>(im.tile_width),
                                            im.archive_width - x));
        t.height = static_cast<uint16_t>(min(static_cast<uint64_t>(im.tile_height),
                                             im.archive_height - y));
        t.row0 = 0;
        t.row1 = t.height;
        t.col0 = 0;
        t.col1 = t.width;
        t.ox = static_cast<uint32_t>(x);
        t.oy = static_cast<uint32_t>(y);
        const uint64_t esize = (f.flags & TSK_F32) ? 4 : 2;
        t.dst = im.out + y * im.out_pitch + x * esize;
        t.pitch = im.out_pitch;
        t.flags = static_cast<uint8_t>(f.flags | TSK_TRUSTED | TSK_UNPARSED |
                                       (l == 0 ? TSK_FIRST : 0));
        const bool class_width = t.width == 64 || t.width == 128 || t.width == 256;
        if (class_width && ((t.dst | t.pitch) & 15u) == 0) {
            t.flags |= TSK_FULL;
        }
        if (l == 0) {
            const uint32_t *head = reinterpret_cast<const uint32_t *>(f.src);
            uint32_t diff = 0;
            for (int k = 0; k < 16; ++k) {
                diff |= head[k] ^ f.header[k];
            }
            t.reserved = diff != 0 ? 1 : 0;
        }
        return t;
    }
    __device__ uint32_t image_of(uint32_t g) const {
        uint32_t r = 0;
        while (r + 1 < batch->count && g >= batch->files[r].task_end) {
            ++r;
        }
        return r;
    }
    __device__ const tsk_decode_image &image(uint32_t i) const {
        return batch->files[i].image;
    }
    __device__ void calibration(const tsk_decode_task &, StageHeader &h) const {
        h.offset = 0.0f; // plain decode only
        h.gain = 1.0f;
        h.opitch = h.gpitch = 0;
        h.omap = h.gmap = 0;
    }
    __device__ uint64_t result_bytes(const tsk_decode_task &t) const {
        return batch->files[t.image].image.result_bytes;
    }
};

// Producer: stages one task into stage s.
template <typename Sh, typename Source>
__device__ void stage_task(Sh &sh, uint32_t s, const tsk_decode_task &t, const Source &source,
                           const tsk_row_start *rowtab) {
    StageHeader &h = sh.header[s];
    uint64_t src = t.src;
    uint32_t words = static_cast<uint32_t>(t.words_or_tile);
    uint32_t mode = t.mode;
    uint32_t state = kStageOk;
    if constexpr (Source::kTrusted) {
        if (t.flags & TSK_TRUSTED) {
            const tsk_decode_image &im = source.image(t.image);
            const bool unparsed = (t.flags & TSK_UNPARSED) != 0;
            uint32_t produced_status = 0;
            uint64_t end = im.capacity; // unparsed: the file size
            if (!unparsed) {
                const volatile tsk_result *producer =
                    reinterpret_cast<const volatile tsk_result *>(im.encoder_result);
                produced_status = producer->status;
                const uint64_t produced_bytes = producer->bytes_written;
                end = produced_bytes < im.capacity ? produced_bytes : im.capacity;
            }
            if (produced_status != 0) {
                state = kStageSkip;
            } else {
                // The archive is only 4-byte aligned: read the entry as 32-bit words.
                const uint32_t *e = reinterpret_cast<const uint32_t *>(t.src + 64 +
                                                                       32 * t.words_or_tile);
                const uint32_t e0 = e[0], e1 = e[1];
                const uint64_t offset = e[2] | (static_cast<uint64_t>(e[3]) << 32);
                const uint64_t length = e[4] | (static_cast<uint64_t>(e[5]) << 32);
                const uint32_t ew = e1 & 0xffffu, eh = e1 >> 16;
                const uint64_t s_bytes = (t.flags & TSK_F32) ? 4 : 2;
                const uint64_t raw =
                    (static_cast<uint64_t>(t.width) * t.height * s_bytes + 3) / 4 * 4;
                mode = e0 & 0xffu;
                bool bad = mode > TSK_PREDICT || ew != t.width || eh != t.height ||
                           offset % 4 != 0 || length % 4 != 0 || length == 0 || length > raw ||
                           offset > end || length > end - offset;
                if (unparsed) {
                    // The host parser's other index rules (parser.cpp check_index, after
                    // reference src/cpu/parser.cpp:86-126): reserved bytes zero, RAW and
                    // CONSTANT lengths exact, payloads chained from the end of the index to the
                    // end of the file; and the header the host checked.
                    const uint64_t tile = t.words_or_tile;
                    uint64_t expected = 64 + 32ull * im.tile_count;
                    if (tile != 0) {
                        expected = (e[-6] | (static_cast<uint64_t>(e[-5]) << 32)) +
                                   (e[-4] | (static_cast<uint64_t>(e[-3]) << 32));
                    }
                    bad = bad || (e0 >> 8) != 0 || e[6] != 0 || e[7] != 0 || offset != expected ||
                          (mode == TSK_RAW && length != raw) ||
                          (mode == TSK_CONSTANT && length != 4) ||
                          (tile + 1 == im.tile_count && !bad && offset + length != end) ||
                          t.reserved != 0;
                }
                if (bad) {
                    state = kStageMalformed;
                } else {
                    src = t.src + offset;
                    words = static_cast<uint32_t>(length / 4);
                }
            }
        }
    }
    const uint32_t shift = static_cast<uint32_t>(src & 15u);
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
        for (uint64_t p = b > a ? b : a; p < end; p += 4) {
            cp_async4(base + (p - src), reinterpret_cast<const void *>(p));
            async_words = true;
        }
        if (async_words) {
            cp_async_arrive(&sh.full[s]);
        }
        const uint32_t body = b > a ? static_cast<uint32_t>(b - a) : 0u;
        const bool parsed_rows = !(t.flags & TSK_TRUSTED) && mode == TSK_PREDICT;
        const uint32_t row_bytes = parsed_rows ? (t.height * 2u + 15u) & ~15u : 0u;
        const uint32_t tx = body + row_bytes;
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
    if (t.flags & TSK_CALIBRATED) {
        source.calibration(t, h);
    }
    h.shift = shift;
    h.words = words;
    h.mode = mode;
    h.state = state;
    mbar_arrive(&sh.full[s]);
}

// Decodes the tile staged in stage s with the RW warps of this thread's group (slot: this
// warp's index in it), then writes the tile's result-record updates (lead thread). Release: the
// stage is handed back through its empty barrier (producer-warp mode); self-staging groups
// reuse their stages themselves.
template <uint32_t Paths, uint32_t RW, uint32_t G16, uint32_t NR, bool Release, uint32_t Groups,
          typename Sh, typename Source>
__device__ __forceinline__ void consume_tile(Sh &sh, uint32_t s, const Source &source,
                                             tsk_result *results, uint32_t one, uint32_t top,
                                             bool lead, uint32_t slot, uint32_t group) {
    const uint32_t lane = threadIdx.x % 32;
    const StageHeader &h = sh.header[s];
    const tsk_decode_task t = h.task;
    const uint32_t state = h.state, hmode = h.mode;
    const uint32_t *payload = reinterpret_cast<const uint32_t *>(sh.payload[s] + h.shift);
    const bool f32 = (t.flags & TSK_F32) != 0;
    const bool calibrated = (t.flags & TSK_CALIBRATED) != 0;
    const bool trusted = (t.flags & TSK_TRUSTED) != 0;
    const bool unparsed = (t.flags & TSK_UNPARSED) != 0;
    bool ok = state == kStageOk;
    if (trusted && ok && (hmode == TSK_PREDICT || unparsed)) {
        auto sync = [&]() {
            if constexpr (RW == 1) {
                __syncwarp();
            } else {
                group_sync<Groups>(group, RW * 32);
            }
        };
        if (lead) {
            bool valid;
            if (hmode == TSK_PREDICT) {
                valid = chain_rows(payload, h.words, t.width, t.height, f32, sh.rows[s]);
            } else if (hmode == TSK_RAW) {
                // The bytes after the last sample are zero.
                const uint32_t tail = (static_cast<uint32_t>(t.width) * t.height * 2u) % 4u;
                valid = f32 || tail == 0 || (payload[h.words - 1] >> 16) == 0;
            } else {
                // A uint16 constant fills the low half of its word.
                valid = f32 || (payload[0] >> 16) == 0;
            }
            sh.valid[s] = valid;
            sh.rowfail[s] = 0;
        }
        sync();
        ok = sh.valid[s] != 0; // read by every thread before any writes rowfail
        if (ok && hmode == TSK_PREDICT) {
            // The rows' own checks, one row per thread of the group.
            for (uint32_t r = slot * 32 + lane; r < t.height; r += RW * 32) {
                if (!row_ok(payload, sh.rows[s][r], t.width, f32, unparsed)) {
                    sh.rowfail[s] = 1;
                }
            }
            sync();
            ok = sh.rowfail[s] == 0;
        }
    }
    if (ok) {
        Ctx x;
        x.out = reinterpret_cast<uint8_t *>(t.dst);
        x.pitch = t.pitch;
        x.w = t.width;
        x.row0 = t.row0;
        x.row1 = t.row1;
        x.col0 = t.col0;
        x.col1 = t.col1;
        x.full = (t.flags & TSK_FULL) != 0;
        x.one = one;
        x.top = top;
        x.slot = slot;
        x.omap = x.gmap = nullptr;
        x.opitch = x.gpitch = 0;
        x.offset = 0.0f;
        x.gain = 1.0f;
        if (calibrated) {
            x.offset = h.offset;
            x.gain = h.gain;
            x.opitch = h.opitch;
            x.gpitch = h.gpitch;
            x.omap = reinterpret_cast<const uint8_t *>(h.omap);
            x.gmap = reinterpret_cast<const uint8_t *>(h.gmap);
        }
        const uint16_t *rows = sh.rows[s];
        if constexpr ((Paths & kU16) && (Paths & kPlain)) {
            if (!f32 && !calibrated) {
                decode_tile<RW, G16, false, false, NR>(x, payload, rows, hmode);
            }
        }
        if constexpr ((Paths & kF32) && (Paths & kPlain)) {
            if (f32 && !calibrated) decode_tile<RW, G16, true, false, NR>(x, payload, rows, hmode);
        }
        if constexpr ((Paths & kU16) && (Paths & kCal)) {
            if (!f32 && calibrated) decode_tile<RW, G16, false, true, NR>(x, payload, rows, hmode);
        }
        if constexpr ((Paths & kF32) && (Paths & kCal)) {
            if (f32 && calibrated) decode_tile<RW, G16, true, true, NR>(x, payload, rows, hmode);
        }
    }
    if constexpr (Release) {
        __syncwarp();
        if (lane == 0) {
            mbar_arrive(&sh.empty[s]);
        }
    }
    if (lead) {
        bool counted = false;
        if constexpr (Source::kTrusted) {
            if (trusted) {
                counted = true;
                const tsk_decode_image &im = source.image(t.image);
                if (state == kStageMalformed || (state == kStageOk && !ok)) {
                    fail(results, t.image, 5u); // malformed_data
                }
                // Completion count: the last task of the image writes the final record. A
                // source with per-CTA tallies (FileSource) adds them once per CTA instead.
                uint32_t done = 0;
                if constexpr (Source::kLocalCounts) {
                    atomicAdd(&source.done[t.image], 1u);
                } else {
                    __threadfence();
                    done = atomicAdd(&results[t.image].reserved, 1u) + 1;
                }
                if (!Source::kLocalCounts && done == im.tile_count) {
                    __threadfence();
                    uint32_t status =
                        *reinterpret_cast<volatile uint32_t *>(&results[t.image].status);
                    const uint32_t produced =
                        im.encoder_result != 0
                            ? reinterpret_cast<const volatile tsk_result *>(im.encoder_result)
                                  ->status
                            : 0u;
                    if (produced != 0) {
                        status = produced;
                    }
                    results[t.image].reserved = 0;
                    results[t.image].bytes_written = status == 0 ? im.result_bytes : 0;
                    results[t.image].status = status;
                }
            }
        }
        if (!counted && (t.flags & TSK_FIRST)) {
            results[t.image].status = 0;
            results[t.image].reserved = 0;
            results[t.image].bytes_written = source.result_bytes(t);
        }
    }
}

// The persistent loop over a task source: CW consumer warps, G16 columns per lane for uint16
// rows. The consumers form CW / RW groups of RW warps; group g decodes this CTA's tiles g,
// g + CW / RW, ..., each of its warps a slice of the tile's rows, and the group releases the
// tile's stage. RW = CW: every warp works on every tile; smaller groups run a tile's set-up
// fewer times per tile.
//
// Dyn: the device work queue. Instead of the static stride, the producer claims chunks of kChunk
// consecutive tasks from a counter in device memory (cleared before the launch), one chunk
// ahead, so CTAs that drew cheap tiles take more of them; after the last task it stages one end
// marker per consumer group.
template <uint32_t MaxPayload, uint32_t Stages, uint32_t Paths, uint32_t CW, uint32_t G16,
          uint32_t NR, uint32_t RW, bool Dyn = false, bool Reserve = false, typename Source>
__device__ __forceinline__ void decode_body(Source &source, const tsk_row_start *rowtab,
                                            tsk_result *results, uint32_t one, uint32_t top) {
    using Sh = Shared<MaxPayload, Stages>;
    constexpr uint32_t kConsumers = CW * 32;
    constexpr uint32_t kGroups = CW / RW;
    static_assert(CW % RW == 0, "groups of equal size");
    extern __shared__ __align__(128) uint8_t smem_raw[];
    Sh &sh = *reinterpret_cast<Sh *>(smem_raw);
    const uint32_t warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < Stages; ++s) {
            mbar_init(&sh.full[s], 1);
            mbar_init(&sh.empty[s], RW);
        }
        fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        griddep_launch_dependents();
    }
    const uint32_t ntasks = source.ntasks;
    const uint32_t mine = blockIdx.x < ntasks ? (ntasks - 1 - blockIdx.x) / gridDim.x + 1 : 0;

    if (warp == CW) {
        // Producer warp: lane 0 issues everything. The next task record is loaded before
        // waiting for a free stage, so its latency overlaps the consumers' work. Task records
        // are the plan's (or the server's) own tables, written before any launch, and so are
        // parsed payloads: a parsed source must stay byte-identical to the one validated when
        // the plan was prepared, for as long as the plan is used (docs/api.md, "Batch plans and
        // ownership"). Both are therefore read without waiting for the stream's previous grid,
        // so the first stages fill while that grid finishes. Encoder output may be that grid's
        // product: the first trusted task waits for it (griddep_wait) before it is staged.
        if (lane != 0) {
            return;
        }
        if constexpr (Dyn) {
            constexpr uint32_t kChunk = 4;
            uint32_t g = atomicAdd(source.claims, kChunk);
            uint32_t end = g + kChunk < ntasks ? g + kChunk : ntasks;
            uint32_t ahead = g < ntasks ? atomicAdd(source.claims, kChunk) : ntasks;
            tsk_decode_task t{};
            if (g < ntasks) {
                t = source.task(g);
            }
            bool waited = false;
            uint32_t i = 0;
            for (; g < ntasks; ++i) {
                const uint32_t s = i % Stages;
                uint32_t ng = g + 1;
                if (ng >= end) {
                    ng = ahead;
                    end = ng + kChunk < ntasks ? ng + kChunk : ntasks;
                    ahead = ng < ntasks ? atomicAdd(source.claims, kChunk) : ntasks;
                }
                tsk_decode_task next{};
                if (ng < ntasks) {
                    next = source.task(ng);
                }
                if (i >= Stages && !mbar_wait(&sh.empty[s], ((i / Stages) - 1) & 1u)) {
                    return; // consumers stopped; they have reported the timeout
                }
                if (!waited && (t.flags & TSK_TRUSTED)) {
                    griddep_wait();
                    waited = true;
                }
                stage_task(sh, s, t, source, rowtab);
                t = next;
                g = ng;
            }
            for (uint32_t k = 0; k < kGroups; ++k, ++i) {
                const uint32_t s = i % Stages;
                if (i >= Stages && !mbar_wait(&sh.empty[s], ((i / Stages) - 1) & 1u)) {
                    return;
                }
                sh.header[s].state = kStageEnd;
                mbar_arrive(&sh.full[s]);
            }
            return;
        }
        tsk_decode_task t{};
        if (mine != 0) {
            t = source.task(blockIdx.x);
        }
        bool waited = false;
        for (uint32_t i = 0; i < mine; ++i) {
            const uint32_t s = i % Stages;
            tsk_decode_task next{};
            if (i + 1 < mine) {
                next = source.task(blockIdx.x + (i + 1) * gridDim.x);
            }
            if (i >= Stages) {
                const bool freed = RW < CW ? mbar_wait_backoff(&sh.empty[s], ((i / Stages) - 1) & 1u)
                                           : mbar_wait(&sh.empty[s], ((i / Stages) - 1) & 1u);
                if (!freed) {
                    return; // consumers stopped; they have reported the timeout
                }
            }
            if (!waited && (t.flags & TSK_TRUSTED)) {
                griddep_wait();
                waited = true;
            }
            stage_task(sh, s, t, source, rowtab);
            t = next;
        }
        return;
    }

    // Consumers write outputs and result records, which the stream's previous grid may still
    // be reading or writing.
    griddep_wait();
    // The thread that walks trusted rows and writes result records for this group's tiles.
    const uint32_t group = warp / RW, slot = warp % RW;
    const bool lead = lane == 0 && slot == 0;
    uint32_t last_image = 0; // Dyn: the image a timeout is reported on
    for (uint32_t i = group; Dyn || i < mine; i += kGroups) {
        const uint32_t s = i % Stages;
        if (!mbar_wait(&sh.full[s], (i / Stages) & 1u)) {
            if (lead) {
                fail(results, Dyn ? last_image : source.image_of(blockIdx.x + i * gridDim.x),
                     9u); // cuda_error
            }
            break;
        }
        if constexpr (Dyn) {
            if (sh.header[s].state == kStageEnd) {
                break;
            }
            last_image = sh.header[s].task.image;
        }
        consume_tile<Paths, RW, G16, NR, true, Reserve ? 0u : kGroups>(sh, s, source, results, one,
                                                                        top, lead, slot,
                                               group);
    }
    if constexpr (Source::kLocalCounts) {
        // Every consumer warp is past its last tile (or gave up on a stage): the CTA's tallies
        // are final. Barrier 1 + kGroups is used by nothing else.
        named_sync<1 + kGroups>(kConsumers);
        if (threadIdx.x < source.batch->count) {
            source.flush(threadIdx.x, results);
        }
    }
}

// The persistent loop without a producer warp: CW consumer warps in CW / RW groups, each group
// staging its own tiles into two stages of its own (stages 2g and 2g + 1) and decoding them in
// turn, so no group waits on another's progress. Group g takes this CTA's tiles g, g + CW / RW,
// ...; its k-th tile uses stage 2g + (k & 1). After a tile is decoded the group synchronises,
// and the group's lead thread restages that stage with the group's tile after next while the
// other stage, already loaded, is decoded. Each lead thread prefetches the task record of the
// tile it will stage next. Stages must equal 2 * CW / RW.
template <uint32_t MaxPayload, uint32_t Stages, uint32_t Paths, uint32_t CW, uint32_t G16,
          uint32_t NR, uint32_t RW, typename Source>
__device__ __forceinline__ void decode_body_self(Source &source, const tsk_row_start *rowtab,
                                                 tsk_result *results, uint32_t one,
                                                 uint32_t top) {
    using Sh = Shared<MaxPayload, Stages>;
    constexpr uint32_t kGroups = CW / RW;
    static_assert(CW % RW == 0 && Stages == 2 * kGroups, "two stages per group");
    extern __shared__ __align__(128) uint8_t smem_raw[];
    Sh &sh = *reinterpret_cast<Sh *>(smem_raw);
    const uint32_t warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const uint32_t group = warp / RW, slot = warp % RW;
    const bool lead = lane == 0 && slot == 0;
    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < Stages; ++s) {
            mbar_init(&sh.full[s], 1);
        }
        fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        griddep_launch_dependents();
    }
    const uint32_t ntasks = source.ntasks;
    const uint32_t mine = blockIdx.x < ntasks ? (ntasks - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    // This group's k-th tile is the CTA's tile group + k * kGroups.
    const uint32_t count = group < mine ? (mine - 1 - group) / kGroups + 1 : 0;
    auto queue_index = [&](uint32_t k) { return blockIdx.x + (group + k * kGroups) * gridDim.x; };
    auto sync_group = [&]() {
        if constexpr (RW == 1) {
            __syncwarp();
        } else {
            tsk::group_sync<kGroups>(group, RW * 32);
        }
    };
    // Task records and parsed payloads are staged before waiting for the stream's previous
    // grid (see decode_body); encoder output, outputs and results are touched after it.
    tsk_decode_task next{};
    if (lead && count > 0) {
        next = source.task(queue_index(0));
    }
    if (lead) {
        for (uint32_t k = 0; k < 2 && k < count; ++k) {
            const tsk_decode_task t = next;
            if (k + 1 < count) {
                next = source.task(queue_index(k + 1));
            }
            if (t.flags & TSK_TRUSTED) {
                griddep_wait();
            }
            stage_task(sh, 2 * group + k, t, source, rowtab);
        }
    }
    griddep_wait();
    for (uint32_t k = 0; k < count; ++k) {
        const uint32_t s = 2 * group + (k & 1u);
        if (!mbar_wait(&sh.full[s], (k >> 1) & 1u)) {
            if (lead) {
                fail(results, source.image_of(queue_index(k)), 9u); // cuda_error
            }
            return;
        }
        consume_tile<Paths, RW, G16, NR, false, kGroups>(sh, s, source, results, one, top, lead, slot,
                                                group);
        if (k + 2 < count) {
            sync_group(); // every warp of the group is done with stage s
            if (lead) {
                const tsk_decode_task t = next;
                if (k + 3 < count) {
                    next = source.task(queue_index(k + 3));
                }
                stage_task(sh, s, t, source, rowtab);
            }
        }
    }
}

// A planned queue (every plan and mixed batch); MinBlocks resident CTAs per SM.
// Reserve: the kernel reserves all sixteen named barriers (named_sync_any), which holds an SM
// to four resident CTAs; uint16 shape 13 measured fastest so (faster than with five, and than
// four enforced by padded shared memory).
template <uint32_t MaxPayload, uint32_t Stages, uint32_t Paths, uint32_t CW, uint32_t G16,
          uint32_t MinBlocks, uint32_t NR, uint32_t RW, bool Self, bool Dyn, bool Reserve>
__global__ void __launch_bounds__(threads_of(CW, Self), MinBlocks)
    decode_kernel(const tsk_decode_task *__restrict__ tasks, uint32_t ntasks,
                  const tsk_decode_image *__restrict__ images,
                  const tsk_row_start *__restrict__ rowtab, tsk_result *results, uint32_t one,
                  uint32_t top, uint32_t *claims) {
    TableSource source{tasks, images, ntasks, claims};
    if constexpr (Self) {
        decode_body_self<MaxPayload, Stages, Paths, CW, G16, NR, RW>(source, rowtab, results, one,
                                                                      top);
    } else {
        decode_body<MaxPayload, Stages, Paths, CW, G16, NR, RW, Dyn, Reserve>(source, rowtab,
                                                                               results, one, top);
    }
}

// A serving batch: the requests arrive in the parameter block.
template <uint32_t MaxPayload, uint32_t Stages, uint32_t Paths, uint32_t CW, uint32_t G16,
          uint32_t MinBlocks, uint32_t NR = 0, uint32_t RW = CW>
__global__ void __launch_bounds__(threads_of(CW), MinBlocks)
    serve_kernel(const __grid_constant__ tsk_serve_batch batch,
                 const tsk_serve_archive *__restrict__ archives,
                 const tsk_row_start *__restrict__ rowtab, tsk_result *results, uint32_t one,
                 uint32_t top) {
    ServeSource source{&batch, archives, batch.ntasks, 0};
    decode_body<MaxPayload, Stages, Paths, CW, G16, NR, RW>(source, rowtab, results, one, top);
}

// A batch of unparsed files: the files arrive in the parameter block.
template <uint32_t MaxPayload, uint32_t Stages, uint32_t Paths, uint32_t CW, uint32_t G16,
          uint32_t MinBlocks, uint32_t NR, uint32_t RW>
__global__ void __launch_bounds__(threads_of(CW), MinBlocks)
    file_kernel(const __grid_constant__ tsk_file_batch batch, tsk_result *results, uint32_t one,
                uint32_t top) {
    __shared__ uint32_t done[TSK_FILE_MAX_BATCH];
    if (threadIdx.x < TSK_FILE_MAX_BATCH) {
        done[threadIdx.x] = 0; // ordered before use by decode_body's first __syncthreads
    }
    FileSource source{&batch, batch.ntasks, 0, done};
    decode_body<MaxPayload, Stages, Paths, CW, G16, NR, RW>(source, nullptr, results, one, top);
}

using KernelFn = void (*)(const tsk_decode_task *, uint32_t, const tsk_decode_image *,
                          const tsk_row_start *, tsk_result *, uint32_t, uint32_t, uint32_t *);

struct Variant {
    KernelFn fn;
    size_t smem;
    uint32_t threads;
    bool dynamic; // claims tasks from the work-queue counter (cleared before each launch)
};

// Kernel instances: uint16-only plans stage 8 KiB tiles (four stages), plans with FP32 stage
// 16 KiB tiles (three stages); the calibrated and plain paths are separate instances so that a
// plan's kernel carries only the code (and registers) it needs. The plain uint16 path, the
// headline one, comes in four shapes (consumer warps x columns per lane) for the tuner.
template <uint32_t MaxPayload, uint32_t Stages, uint32_t Paths, uint32_t CW = 8,
          uint32_t G16 = 8, uint32_t MinBlocks = 3, uint32_t NR = 0, uint32_t RW = CW,
          bool Self = false, bool Dyn = false, bool Reserve = false>
Variant make() {
    return {decode_kernel<MaxPayload, Stages, Paths, CW, G16, MinBlocks, NR, RW, Self, Dyn, Reserve>,
            sizeof(Shared<MaxPayload, Stages>), threads_of(CW, Self), Dyn};
}

// Shapes of the plain uint16 instance (consumer warps x uint16 columns per lane, stages,
// resident CTAs per SM in the launch bounds): 0 = 8 x 8, 4 stages, 4; 1 = 8 x 16, 4, 3;
// 2 = 4 x 16, 4, 5; 3 = 4 x 8, 4, 6; 4 = 4 x 16, 4, 6 (64 registers); 5 = 4 x 16, 3, 7 (56
// registers); 6 = 4 x 32, 4, 3; 7 = 4 x 32, 4, 4; 8-11 single-pass rows with one or two rows per
// lane; 12-13 warps in groups of one or two per tile (13: pairs, four CTAs per SM); 14-17
// without a producer warp (each group stages its own tiles; 15, the default: pairs, two stages
// each, up to six CTAs per SM); 18 = 13 with the device work queue.
// The plain mixed uint16 + FP32 instance has twelve: 0 = 8 x 8, 3 stages of 16 KiB, 3 CTAs;
// 1 = 4 x 16, 2 stages, 5 CTAs; 2 = 4 x 16, 3, 4; 3 = 4 x 8, 2, 6 (two stages leave shared
// memory for more resident CTAs); 4-7 variants of them with single-pass rows or warp pairs;
// 8 and 9 = 5 and 6 with the device work queue; 10 and 11 without a producer warp.
// The other instances have shapes 0 and 2 (odd shapes map to 0, even ones to 2), and
// single-pass rows from shape 8 on (a variant without a producer warp was slower for the fused
// FP32 calibration: 55.8 against 51.8 us).
Variant select(uint32_t paths, uint32_t shape) {
    const bool f32 = paths & kF32, u16 = paths & kU16, plain = paths & kPlain, c = paths & kCal;
    const bool narrow = shape % 2 == 0 && shape != 0; // four consumer warps
    if (!f32) {
        if (plain && !c) {
            switch (shape) {
            case 1:
                return make<8192, 4, kU16 | kPlain, 8, 16, 3>();
            case 2:
                return make<8192, 4, kU16 | kPlain, 4, 16, 5>();
            case 3:
                return make<8192, 4, kU16 | kPlain, 4, 8, 6>();
            case 4:
                return make<8192, 4, kU16 | kPlain, 4, 16, 6>();
            case 5:
                return make<8192, 3, kU16 | kPlain, 4, 16, 7>();
            case 6:
                return make<8192, 4, kU16 | kPlain, 4, 32, 3>();
            case 7:
                return make<8192, 4, kU16 | kPlain, 4, 32, 4>();
            case 8:
                return make<8192, 4, kU16 | kPlain, 4, 16, 5, 1>();
            case 9:
                return make<8192, 4, kU16 | kPlain, 4, 16, 4, 2>();
            case 10:
                return make<8192, 4, kU16 | kPlain, 4, 16, 5, 2>();
            case 11:
                return make<8192, 4, kU16 | kPlain, 4, 8, 5, 2>();
            case 12:
                return make<8192, 5, kU16 | kPlain, 4, 16, 4, 1, 1>();
            case 13: // four CTAs per SM (all named barriers reserved)
                return make<8192, 4, kU16 | kPlain, 4, 16, 5, 1, 2, false, false, true>();
            case 14:
                return make<8192, 4, kU16 | kPlain, 4, 16, 5, 1, 2, true>();
            case 15:
                return make<8192, 4, kU16 | kPlain, 4, 16, 6, 1, 2, true>();
            case 16:
                return make<8192, 4, kU16 | kPlain, 4, 16, 4, 2, 2, true>();
            case 17:
                return make<8192, 8, kU16 | kPlain, 4, 16, 3, 1, 1, true>();
            case 18: // shape 13 with the device work queue
                return make<8192, 4, kU16 | kPlain, 4, 16, 5, 1, 2, false, true>();
            default:
                return make<8192, 4, kU16 | kPlain, 8, 8, 4>();
            }
        }
        if (c && !plain) {
            if (shape >= 8) return make<8192, 4, kU16 | kCal, 4, 16, 4, 1>();
            return narrow ? make<8192, 4, kU16 | kCal, 4, 16, 4>() : make<8192, 4, kU16 | kCal>();
        }
        if (shape >= 8) return make<8192, 4, kU16 | kPlain | kCal, 4, 16, 4, 1>();
        return make<8192, 4, kU16 | kPlain | kCal>();
    }
    if (!u16) {
        if (plain && !c) {
            if (shape >= 8) return make<16384, 3, kF32 | kPlain, 4, 16, 4, 1>();
            return narrow ? make<16384, 3, kF32 | kPlain, 4, 16, 4>()
                          : make<16384, 3, kF32 | kPlain>();
        }
        if (c && !plain) {
            if (shape >= 8) return make<16384, 3, kF32 | kCal, 4, 16, 4, 1>();
            return narrow ? make<16384, 3, kF32 | kCal, 4, 16, 4>() : make<16384, 3, kF32 | kCal>();
        }
    } else if (plain && !c) {
        // Mixed uint16 and FP32 archives, plain decode (no calibrated code in the instance).
        switch (shape) {
        case 1:
            return make<16384, 2, kU16 | kF32 | kPlain, 4, 16, 5>();
        case 3:
            return make<16384, 2, kU16 | kF32 | kPlain, 4, 8, 6>();
        case 4: // warp pairs per tile, two stages per pair
            return make<16384, 4, kU16 | kF32 | kPlain, 4, 16, 3, 1, 2>();
        case 5: // shape 1 with the single-pass uint16 rows
            return make<16384, 2, kU16 | kF32 | kPlain, 4, 16, 5, 1>();
        case 6: // shape 2 with the single-pass uint16 rows
            return make<16384, 3, kU16 | kF32 | kPlain, 4, 16, 4, 1>();
        case 7: // shape 5 with six CTAs per SM
            return make<16384, 2, kU16 | kF32 | kPlain, 4, 16, 6, 1>();
        case 8: // shape 5 with the device work queue
            return make<16384, 2, kU16 | kF32 | kPlain, 4, 16, 5, 1, 4, false, true>();
        case 9: // shape 6 with the device work queue
            return make<16384, 3, kU16 | kF32 | kPlain, 4, 16, 4, 1, 4, false, true>();
        case 10: // no producer warp: one group of four warps staging its own tiles
            return make<16384, 2, kU16 | kF32 | kPlain, 4, 16, 6, 1, 4, true>();
        case 11: // no producer warp: two pairs, each staging its own tiles
            return make<16384, 4, kU16 | kF32 | kPlain, 4, 16, 3, 1, 2, true>();
        default:
            return narrow ? make<16384, 3, kU16 | kF32 | kPlain, 4, 16, 4>()
                          : make<16384, 3, kU16 | kF32 | kPlain>();
        }
    }
    if (shape >= 8) return make<16384, 3, kU16 | kF32 | kPlain | kCal, 4, 16, 4, 1>();
    return narrow ? make<16384, 3, kU16 | kF32 | kPlain | kCal, 4, 16, 4>()
                  : make<16384, 3, kU16 | kF32 | kPlain | kCal>();
}

using ServeFn = void (*)(tsk_serve_batch, const tsk_serve_archive *, const tsk_row_start *,
                         tsk_result *, uint32_t, uint32_t);

struct ServeVariant {
    ServeFn fn;
    size_t smem;
    uint32_t threads;
};

// Serving instances: uint16 archives (plain and scalar-calibrated requests), and any archives.
ServeVariant select_serve(bool all_u16) {
    if (all_u16) {
        // Eight warps x 8 columns per lane: on ROI-cut tiles it serves faster than the plain
        // decoder's default shape (p99 49 against 72 us at 20k requests/s).
        return {serve_kernel<8192, 4, kU16 | kPlain | kCal, 8, 8, 3>, sizeof(Shared<8192, 4>),
                threads_of(8)};
    }
    return {serve_kernel<16384, 3, kU16 | kF32 | kPlain | kCal, 8, 8, 3>,
            sizeof(Shared<16384, 3>), threads_of(8)};
}

using FileFn = void (*)(tsk_file_batch, tsk_result *, uint32_t, uint32_t);

struct FileVariant {
    FileFn fn;
    size_t smem;
    uint32_t threads;
};

// Unparsed-file instances, plain decode: uint16 files in the default plain uint16 shape (4
// warps x 16 columns in warp pairs, single-pass rows, 4 stages of 8 KiB, 5 CTAs per SM), and
// batches with FP32 files in the mixed batch's shape 5 (two 16 KiB stages, 5 CTAs per SM).
FileVariant select_file(bool any_f32) {
    if (!any_f32) {
        return {file_kernel<8192, 4, kU16 | kPlain, 4, 16, 5, 1, 2>, sizeof(Shared<8192, 4>),
                threads_of(4)};
    }
    return {file_kernel<16384, 2, kU16 | kF32 | kPlain, 4, 16, 5, 1, 4>,
            sizeof(Shared<16384, 2>), threads_of(4)};
}

} // namespace
} // namespace tsk

// Sets the kernel instance's shared-memory limit (which also loads it) and fills in the
// occupancy-derived persistent grid for the plan's path mask and kernel shape.
namespace {

// The occupancy of a kernel instance on a device, found by the first plan that uses the
// instance there: later plans skip the query. Entries are keyed by (device, kernel function).
// The shared-memory attribute is set by every plan, so a device reset cannot leave an instance
// without it.
struct Prepared {
    int device = -1;
    const void *fn = nullptr;
    int per_sm = 0;
    int sms = 0;
};
constexpr int kPreparedSlots = 256;
std::mutex g_prepared_mutex;
Prepared g_prepared[kPreparedSlots];
int g_prepared_count = 0;

} // namespace

// Dynamic shared memory per CTA with which exactly per_sm CTAs of v share an SM when its
// occupancy (`fits` CTAs) is higher: the block scheduler places as many CTAs on an SM as fit,
// so a grid of SMs x per_sm CTAs would otherwise leave SMs empty. Never below v's own need.
size_t residency_smem(const tsk::Variant &v, int per_sm, int fits, int device) {
    if (per_sm >= fits) {
        return v.smem;
    }
    int total = 0, reserved = 0;
    if (cudaDeviceGetAttribute(&total, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device) !=
            cudaSuccess ||
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, device) !=
            cudaSuccess) {
        cudaGetLastError();
        return v.smem;
    }
    // (per_sm + 1) CTAs of this size exceed the SM's shared memory; per_sm still fit.
    const size_t padded = static_cast<size_t>(total / (per_sm + 1) - reserved + 1 + 127) / 128 * 128;
    const size_t smem = padded > v.smem ? padded : v.smem;
    return static_cast<size_t>(per_sm) * (smem + reserved) <= static_cast<size_t>(total) ? smem
                                                                                         : v.smem;
}

// The grid and shared memory of a launch for per_sm resident CTAs per SM (at most the
// occupancy of the instance, `fits`).
void set_residency(tsk_decode_config *config, const tsk::Variant &v, int per_sm, int fits,
                   int sms, uint32_t ntasks, int device) {
    if (per_sm > fits) per_sm = fits;
    if (per_sm < 1) per_sm = 1;
    uint64_t grid = static_cast<uint64_t>(sms) * per_sm;
    if (grid > ntasks) grid = ntasks;
    if (grid < 1) grid = 1;
    config->grid = static_cast<uint32_t>(grid);
    config->per_sm = static_cast<uint32_t>(per_sm);
    config->smem = static_cast<uint32_t>(residency_smem(v, per_sm, fits, device));
}

extern "C" int tsk_decode_prepare(tsk_decode_config *config, uint32_t ntasks, int device) {
    const tsk::Variant v = tsk::select(config->paths, config->shape);
    const void *key = reinterpret_cast<const void *>(v.fn);
    int per_sm = 0, sms = 0;
    {
        std::lock_guard<std::mutex> lock(g_prepared_mutex);
        for (int i = 0; i < g_prepared_count; ++i) {
            if (g_prepared[i].device == device && g_prepared[i].fn == key) {
                per_sm = g_prepared[i].per_sm;
                sms = g_prepared[i].sms;
                break;
            }
        }
    }
    // Any padding set_residency chooses is allowed: the limit is the device's per-block maximum.
    int optin = 0;
    cudaError_t e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(v.fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             optin > static_cast<int>(v.smem) ? optin : static_cast<int>(v.smem));
    if (e != cudaSuccess) return e;
    // The largest shared-memory carveout, so that occupancy is bounded by the instance's own
    // needs and not by the default split between L1 and shared memory.
    e = cudaFuncSetAttribute(v.fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    if (sms == 0) {
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, v.fn, v.threads, v.smem);
        if (e != cudaSuccess) return e;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (e != cudaSuccess) return e;
        std::lock_guard<std::mutex> lock(g_prepared_mutex);
        if (g_prepared_count < kPreparedSlots) {
            g_prepared[g_prepared_count++] = {device, key, per_sm, sms};
        }
    }
    const int fits = per_sm < 1 ? 1 : per_sm;
    set_residency(config, v, fits, fits, sms, ntasks, device);
    config->fits = static_cast<uint32_t>(fits);
    return cudaSuccess;
}

extern "C" int tsk_decode_residency(tsk_decode_config *config, uint32_t per_sm, uint32_t ntasks,
                                    int device) {
    const tsk::Variant v = tsk::select(config->paths, config->shape);
    int sms = 0;
    const cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    set_residency(config, v, static_cast<int>(per_sm), static_cast<int>(config->fits), sms, ntasks,
                  device);
    return cudaSuccess;
}

// Launched as a programmatic dependent of the stream's previous grid: this grid's CTAs may
// start (barrier set-up, task records, parsed payloads) while that grid finishes, and wait for
// it before reading encoder output or touching outputs and results (decode_body).
extern "C" int tsk_decode_launch(const tsk_decode_task *tasks, uint32_t ntasks,
                                 const tsk_decode_image *images, const tsk_row_start *rows,
                                 tsk_result *results, tsk_decode_config config,
                                 uint32_t *claims, cudaStream_t stream) {
    if (ntasks == 0) return cudaSuccess;
    const tsk::Variant v = tsk::select(config.paths, config.shape);
    if (v.dynamic) {
        const cudaError_t e = cudaMemsetAsync(claims, 0, sizeof(uint32_t), stream);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(config.grid);
    cfg.blockDim = dim3(v.threads);
    cfg.dynamicSmemBytes = config.smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, v.fn, tasks, ntasks, images, rows, results, 1u, 0x80000000u,
                              claims);
}

// A CUDA graph of one execution: a clear of the result records when the plan has trusted images
// (their completion is counted in the records), then the decode kernel node.
extern "C" int tsk_decode_graph(const tsk_decode_task *tasks, uint32_t ntasks,
                                const tsk_decode_image *images, const tsk_row_start *rows,
                                tsk_result *results, uint32_t result_count, int clear_results,
                                tsk_decode_config config, uint32_t *claims,
                                cudaGraph_t *graph_out, cudaGraphExec_t *exec_out) {
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaGraphCreate(&graph, 0);
    if (e != cudaSuccess) return e;
    const tsk::Variant v = tsk::select(config.paths, config.shape);
    cudaGraphNode_t before[2] = {nullptr, nullptr}, kernel = nullptr;
    size_t nbefore = 0;
    auto clear = [&](void *dst, size_t bytes) {
        cudaMemsetParams m{};
        m.dst = dst;
        m.value = 0;
        m.elementSize = 1;
        m.width = bytes;
        m.height = 1;
        m.pitch = 0;
        return cudaGraphAddMemsetNode(&before[nbefore++], graph, nullptr, 0, &m);
    };
    if (clear_results && result_count != 0) {
        e = clear(results, sizeof(tsk_result) * result_count);
    }
    if (e == cudaSuccess && v.dynamic && ntasks != 0) {
        e = clear(claims, sizeof(uint32_t));
    }
    if (e == cudaSuccess && ntasks != 0) {
        uint32_t one = 1u, top = 0x80000000u;
        void *args[] = {&tasks, &ntasks, &images, &rows, &results, &one, &top, &claims};
        cudaKernelNodeParams k{};
        k.func = reinterpret_cast<void *>(v.fn);
        k.gridDim = dim3(config.grid);
        k.blockDim = dim3(v.threads);
        k.sharedMemBytes = config.smem;
        k.kernelParams = args;
        k.extra = nullptr;
        e = cudaGraphAddKernelNode(&kernel, graph, nbefore != 0 ? before : nullptr, nbefore, &k);
    }
    if (e == cudaSuccess) {
        e = cudaGraphInstantiate(exec_out, graph, 0);
    }
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return e;
    }
    *graph_out = graph;
    return cudaSuccess;
}

extern "C" int tsk_serve_prepare(int all_u16, int device, uint32_t *grid) {
    const tsk::ServeVariant v = tsk::select_serve(all_u16 != 0);
    cudaError_t e = cudaFuncSetAttribute(v.fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(v.smem));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(v.fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, v.fn, v.threads, v.smem);
    if (e != cudaSuccess) return e;
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    *grid = static_cast<uint32_t>(sms) * static_cast<uint32_t>(per_sm < 1 ? 1 : per_sm);
    return cudaSuccess;
}

extern "C" int tsk_serve_launch(const tsk_serve_batch *batch, const tsk_serve_archive *archives,
                                const tsk_row_start *rows, tsk_result *results, uint32_t grid,
                                int all_u16, cudaStream_t stream) {
    if (batch->ntasks == 0) return cudaSuccess;
    const tsk::ServeVariant v = tsk::select_serve(all_u16 != 0);
    const uint32_t blocks = grid < batch->ntasks ? grid : batch->ntasks;
    v.fn<<<blocks, v.threads, v.smem, stream>>>(*batch, archives, rows, results, 1u, 0x80000000u);
    return cudaGetLastError();
}

extern "C" int tsk_file_prepare(int any_f32, int device, uint32_t *grid) {
    const tsk::FileVariant v = tsk::select_file(any_f32 != 0);
    const void *key = reinterpret_cast<const void *>(v.fn);
    int per_sm = 0, sms = 0;
    {
        std::lock_guard<std::mutex> lock(g_prepared_mutex);
        for (int i = 0; i < g_prepared_count; ++i) {
            if (g_prepared[i].device == device && g_prepared[i].fn == key) {
                per_sm = g_prepared[i].per_sm;
                sms = g_prepared[i].sms;
                break;
            }
        }
    }
    if (sms == 0) {
        cudaError_t e = cudaFuncSetAttribute(v.fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(v.smem));
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(v.fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared);
        if (e != cudaSuccess) return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, v.fn, v.threads, v.smem);
        if (e != cudaSuccess) return e;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (e != cudaSuccess) return e;
        std::lock_guard<std::mutex> lock(g_prepared_mutex);
        if (g_prepared_count < kPreparedSlots) {
            g_prepared[g_prepared_count++] = {device, key, per_sm, sms};
        }
    }
    *grid = static_cast<uint32_t>(sms) * static_cast<uint32_t>(per_sm < 1 ? 1 : per_sm);
    return cudaSuccess;
}

extern "C" int tsk_file_launch(const tsk_file_batch *batch, tsk_result *results, uint32_t grid,
                               int any_f32, cudaStream_t stream) {
    if (batch->count == 0) return cudaSuccess;
    // Validation counts each file's finished tiles in its record: the records start cleared.
    cudaError_t e = cudaMemsetAsync(results, 0, sizeof(tsk_result) * batch->count, stream);
    if (e != cudaSuccess || batch->ntasks == 0) return e;
    const tsk::FileVariant v = tsk::select_file(any_f32 != 0);
    const uint32_t blocks = grid < batch->ntasks ? grid : batch->ntasks;
    v.fn<<<blocks, v.threads, v.smem, stream>>>(*batch, results, 1u, 0x80000000u);
    return cudaGetLastError();
}
