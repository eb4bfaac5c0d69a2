// Single-pass canonical .tsc encoder for sm_100a.
//
// The reference encodes a window with four launches and a library scan: analyze (residuals to
// a 16 KiB-per-tile global workspace), cub::DeviceScan over tile lengths, pack (re-reading the
// input and the residuals) and finish (src/cuda/encoder.cu:62-327). Here one persistent kernel
// does all of it and reads each input pixel once:
//
//  1. a CTA takes the next tile in batch order from an atomic counter, loads its pixels into
//     shared memory and computes the residuals (zigzag mod 2^16 or XOR, encoder.cpp:32-37);
//  2. one warp per row OR-reduces the residuals with shuffles; the row width is the index of
//     the highest set bit (docs/format.md:101), the row costs are scanned with a warp shuffle
//     scan, and the canonical mode is chosen with the tie order RAW < CONSTANT < PREDICT
//     (docs/format.md:103-109, encoder.cpp:69-78);
//  3. the tile's payload offset is the exclusive prefix of the lengths of the earlier tiles of
//     the same image, found by a decoupled look-back over per-tile flags in the workspace
//     (tile i publishes its length at once and its inclusive prefix when known; waits are
//     bounded and report cuda_error instead of hanging);
//  4. the index entry and every payload word are written by exactly one thread, gathering the
//     residuals that overlap the word (encoder.cu:157-173 does the same from global memory);
//  5. the last tile of an image writes the 64-byte header and the image's DeviceResult.
#include "ptx.cuh"
#include "tasks.h"

#include <cstdint>
#include <mutex>

namespace tsk {
namespace {

constexpr uint32_t kThreads = 256;
constexpr uint32_t kWarps = kThreads / 32;
constexpr uint64_t kAggregate = 1ull << 62;
constexpr uint64_t kPrefix = 2ull << 62;
constexpr uint64_t kValue = (1ull << 62) - 1;

struct EncodeShared {
    uint32_t px[TSK_TILE_PIXELS];
    uint32_t res[TSK_TILE_PIXELS]; // res[r * w + c] = residual of column c (c >= 1)
    uint32_t bits[TSK_MAX_ROWS];
    uint32_t row_word[TSK_MAX_ROWS + 1]; // first payload word of each row
    uint64_t offset;                     // absolute file offset of the payload
    uint64_t inclusive;                  // prefix including this tile
    uint64_t tile_id;
    uint32_t mode;
    uint32_t length;
    uint32_t image;
};

template <bool F32> __device__ __forceinline__ uint32_t residual(uint32_t cur, uint32_t prev) {
    if constexpr (F32) {
        return cur ^ prev;
    } else {
        const uint32_t d = (cur - prev) & 0xffffu;
        return d < 32768u ? d * 2u : (65536u - d) * 2u - 1u;
    }
}

__device__ __forceinline__ uint64_t ld_acquire(const uint64_t *p) {
    uint64_t v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(uint64_t *p, uint64_t v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void put_word(uint8_t *file, uint64_t byte, uint32_t v) {
    *reinterpret_cast<uint32_t *>(file + byte) = v;
}

// Word k of a PREDICT row of width w and residual width b: the bits [32 k, 32 k + 32) of the
// packed residuals 1..w-1 (docs/format.md:77).
__device__ __forceinline__ uint32_t packed_word(const uint32_t *res, uint32_t w, uint32_t b,
                                                uint32_t k) {
    if (b == 32) {
        return res[1 + k];
    }
    const uint32_t first_bit = 32 * k;
    const uint32_t count = w - 1;
    const uint32_t j_end = (first_bit + 31) / b;
    const uint32_t last = j_end < count - 1 ? j_end : count - 1;
    uint32_t value = 0;
    for (uint32_t j = first_bit / b; j <= last; ++j) {
        const uint32_t pos = j * b;
        const uint32_t r = res[1 + j];
        value |= pos >= first_bit ? r << (pos - first_bit) : r >> (first_bit - pos);
    }
    return value;
}

template <bool F32>
__device__ void encode_tile(EncodeShared &sh, const tsk_encode_image &im, uint64_t index,
                            uint64_t *flags, uint64_t global_tile, tsk_result *results,
                            uint32_t image) {
    const uint32_t warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const uint64_t x = (index % im.columns) * im.tile_width;
    const uint64_t y = (index / im.columns) * im.tile_height;
    const uint32_t w = static_cast<uint32_t>(im.width - x < im.tile_width ? im.width - x
                                                                          : im.tile_width);
    const uint32_t h = static_cast<uint32_t>(im.height - y < im.tile_height ? im.height - y
                                                                            : im.tile_height);
    constexpr uint32_t s = F32 ? 4 : 2;
    const uint8_t *origin = reinterpret_cast<const uint8_t *>(im.input) + y * im.pitch + x * s;

    // 1. Pixels into shared memory, one warp per row; 16-byte loads when the row allows.
    const bool vec = ((reinterpret_cast<uintptr_t>(origin) | im.pitch | (w * s)) & 15u) == 0;
    for (uint32_t r = warp; r < h; r += kWarps) {
        const uint8_t *line = origin + r * im.pitch;
        uint32_t *dst = sh.px + r * w;
        if (vec) {
            constexpr uint32_t per = 16 / s;
            for (uint32_t c = lane * per; c < w; c += 32 * per) {
                const uint4 v = ld_nc_v4(line + c * s);
                if constexpr (F32) {
                    dst[c] = v.x;
                    dst[c + 1] = v.y;
                    dst[c + 2] = v.z;
                    dst[c + 3] = v.w;
                } else {
                    const uint32_t q[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                    for (uint32_t e = 0; e < 4; ++e) {
                        dst[c + 2 * e] = q[e] & 0xffffu;
                        dst[c + 2 * e + 1] = q[e] >> 16;
                    }
                }
            }
        } else {
            for (uint32_t c = lane; c < w; c += 32) {
                if constexpr (F32) {
                    dst[c] = reinterpret_cast<const uint32_t *>(line)[c];
                } else {
                    dst[c] = reinterpret_cast<const uint16_t *>(line)[c];
                }
            }
        }
    }
    __syncthreads();

    // 2. Residuals, row widths and the constant test.
    const uint32_t first = sh.px[0];
    bool constant = true;
    for (uint32_t r = warp; r < h; r += kWarps) {
        const uint32_t *line = sh.px + r * w;
        uint32_t combined = 0;
        for (uint32_t c = lane; c < w; c += 32) {
            const uint32_t cur = line[c];
            constant = constant && cur == first;
            if (c != 0) {
                const uint32_t z = residual<F32>(cur, line[c - 1]);
                sh.res[r * w + c] = z;
                combined |= z;
            }
        }
#pragma unroll
        for (uint32_t d = 16; d > 0; d >>= 1) {
            combined |= __shfl_xor_sync(0xffffffffu, combined, d);
        }
        if (lane == 0) {
            sh.bits[r] = 32u - __clz(combined);
        }
    }
    const bool uniform = __syncthreads_and(constant) != 0;

    // Row costs in words (descriptor + packed residuals), scanned by warp 0.
    if (warp == 0) {
        uint32_t carry = 0;
        for (uint32_t base = 0; base < h; base += 32) {
            const uint32_t r = base + lane;
            const uint32_t cost = r < h ? 2u + ((w - 1) * sh.bits[r] + 31u) / 32u : 0u;
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

            // 3. Decoupled look-back over the earlier tiles of this image.
            uint64_t *flag = flags + global_tile;
            uint64_t prefix = 0;
            if (index == 0) {
                st_release(flag, kPrefix | length);
            } else {
                st_release(flag, kAggregate | length);
                uint64_t j = global_tile - 1;
                bool timed_out = false;
                for (;;) {
                    uint64_t v = ld_acquire(flags + j);
                    uint32_t spins = 0;
                    while ((v >> 62) == 0 && spins < (1u << 22)) {
                        __nanosleep(64);
                        v = ld_acquire(flags + j);
                        ++spins;
                    }
                    if ((v >> 62) == 0) {
                        timed_out = true;
                        break;
                    }
                    prefix += v & kValue;
                    if ((v >> 62) == 2) {
                        break;
                    }
                    --j;
                }
                if (timed_out) {
                    atomicCAS(&results[image].status, 0u, 9u);
                }
                st_release(flag, kPrefix | (prefix + length));
            }
            const uint64_t base = 64 + 32 * im.tile_count;
            sh.offset = base + prefix;
            sh.inclusive = prefix + length;
        }
    }
    __syncthreads();

    // 4. Index entry and payload, one writer per word.
    uint8_t *file = reinterpret_cast<uint8_t *>(im.output);
    const uint32_t mode = sh.mode, length = sh.length;
    const uint64_t offset = sh.offset;
    if (threadIdx.x < 8) {
        uint32_t v = 0;
        switch (threadIdx.x) {
        case 0: v = mode; break;
        case 1: v = w | (h << 16); break;
        case 2: v = static_cast<uint32_t>(offset); break;
        case 3: v = static_cast<uint32_t>(offset >> 32); break;
        case 4: v = length; break;
        default: v = 0; break;
        }
        put_word(file, 64 + 32 * index + 4 * threadIdx.x, v);
    }
    const uint32_t words = length / 4;
    if (mode == TSK_RAW) {
        const uint32_t count = w * h;
        for (uint32_t k = threadIdx.x; k < words; k += kThreads) {
            uint32_t v;
            if constexpr (F32) {
                v = sh.px[k];
            } else {
                const uint32_t i0 = 2 * k, i1 = 2 * k + 1;
                v = sh.px[i0] | (i1 < count ? sh.px[i1] << 16 : 0u);
            }
            put_word(file, offset + 4ull * k, v);
        }
    } else if (mode == TSK_CONSTANT) {
        if (threadIdx.x == 0) {
            put_word(file, offset, first);
        }
    } else {
        for (uint32_t k = threadIdx.x; k < words; k += kThreads) {
            // Row of word k: the last row starting at or before it.
            uint32_t lo = 0, hi = h;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) / 2;
                if (sh.row_word[mid] <= k) {
                    lo = mid;
                } else {
                    hi = mid;
                }
            }
            const uint32_t local = k - sh.row_word[lo];
            uint32_t v;
            if (local == 0) {
                v = sh.px[lo * w];
            } else if (local == 1) {
                v = sh.bits[lo];
            } else {
                v = packed_word(sh.res + lo * w, w, sh.bits[lo], local - 2);
            }
            put_word(file, offset + 4ull * k, v);
        }
    }

    // 5. The last tile writes the header and the result.
    if (index + 1 == im.tile_count && threadIdx.x < 16) {
        const uint64_t size = 64 + 32 * im.tile_count + sh.inclusive;
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
            // The launcher cleared the records; a look-back timeout may have set cuda_error.
            results[image].bytes_written = size;
        }
    }
}

__global__ void __launch_bounds__(kThreads)
    encode_kernel(const tsk_encode_image *__restrict__ images, uint32_t image_count,
                  uint64_t total_tiles, uint64_t *state, tsk_result *results) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    EncodeShared &sh = *reinterpret_cast<EncodeShared *>(smem_raw);
    uint64_t *counter = state;
    uint64_t *flags = state + 2;
    for (;;) {
        if (threadIdx.x == 0) {
            const uint64_t id = atomicAdd(reinterpret_cast<unsigned long long *>(counter), 1ull);
            sh.tile_id = id < total_tiles ? id : total_tiles;
            // Image owning tile id: the last image whose first tile is at or before it.
            uint32_t lo = 0, hi = image_count;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) / 2;
                if (images[mid].first_tile <= id) {
                    lo = mid;
                } else {
                    hi = mid;
                }
            }
            sh.image = lo;
        }
        __syncthreads();
        const uint64_t id = sh.tile_id;
        const uint32_t image = sh.image;
        if (id >= total_tiles) {
            return;
        }
        const tsk_encode_image &im = images[image];
        const uint64_t index = id - im.first_tile;
        if (im.type == 2) {
            encode_tile<true>(sh, im, index, flags, id, results, image);
        } else {
            encode_tile<false>(sh, im, index, flags, id, results, image);
        }
        __syncthreads();
    }
}

} // namespace
} // namespace tsk

extern "C" uint64_t tsk_encode_state_bytes(uint64_t total_tiles) {
    return 8 * (total_tiles + 2);
}

extern "C" int tsk_encode_prepare(int device) {
    (void)device;
    cudaError_t e = cudaFuncSetAttribute(tsk::encode_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(sizeof(tsk::EncodeShared)));
    if (e != cudaSuccess) return e;
    cudaFuncAttributes attributes;
    return cudaFuncGetAttributes(&attributes, tsk::encode_kernel);
}

extern "C" int tsk_encode_launch(const tsk_encode_image *images, uint32_t image_count,
                                 uint64_t total_tiles, uint32_t any_float, void *state,
                                 tsk_result *results, cudaStream_t stream) {
    (void)any_float;
    if (total_tiles == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(state, 0, tsk_encode_state_bytes(total_tiles), stream);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(results, 0, sizeof(tsk_result) * image_count, stream);
    if (e != cudaSuccess) return e;
    int device = 0, sms = 0, per_sm = 0;
    e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    const size_t smem = sizeof(tsk::EncodeShared);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tsk::encode_kernel, tsk::kThreads,
                                                      smem);
    if (e != cudaSuccess) return e;
    uint64_t grid = static_cast<uint64_t>(sms) * (per_sm > 0 ? per_sm : 1);
    if (grid > total_tiles) grid = total_tiles;
    tsk::encode_kernel<<<static_cast<uint32_t>(grid), tsk::kThreads, smem, stream>>>(
        images, image_count, total_tiles, static_cast<uint64_t *>(state), results);
    return cudaGetLastError();
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

// At most this many tiles per image: 8 bytes of state per tile plus two words, 1 MiB in all.
constexpr uint64_t kStaticStateWords = 131072;

__device__ __align__(256) uint64_t g_encode_scratch[kStaticStateWords];

__global__ void __launch_bounds__(kThreads)
    encode_kernel_static(tsk_encode_image image, uint64_t total_tiles, uint64_t *state,
                         tsk_result *result) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    EncodeShared &sh = *reinterpret_cast<EncodeShared *>(smem_raw);
    uint64_t *counter = state;
    uint64_t *flags = state + 2;
    for (;;) {
        if (threadIdx.x == 0) {
            const uint64_t id = atomicAdd(reinterpret_cast<unsigned long long *>(counter), 1ull);
            sh.tile_id = id < total_tiles ? id : total_tiles;
            sh.image = 0;
        }
        __syncthreads();
        const uint64_t id = sh.tile_id;
        if (id >= total_tiles) {
            return;
        }
        if (image.type == 2) {
            encode_tile<true>(sh, image, id, flags, id, result, 0);
        } else {
            encode_tile<false>(sh, image, id, flags, id, result, 0);
        }
        __syncthreads();
    }
}

// Per-device set-up, done by the first call on each device with that device current.
struct StaticSetup {
    uint64_t *scratch = nullptr; // device address of g_encode_scratch
    uint32_t grid = 0;
};

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
StaticSetup g_setup[kMaxDevices];

cudaError_t static_setup(int device, StaticSetup &out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    StaticSetup &s = g_setup[device];
    if (s.scratch == nullptr) {
        void *address = nullptr;
        // In host code the name g_encode_scratch is a host-side stand-in, not a device address;
        // the runtime returns this device's copy of the array.
        cudaError_t e = cudaGetSymbolAddress(&address, g_encode_scratch);
        if (e != cudaSuccess) return e;
        const size_t smem = sizeof(EncodeShared);
        e = cudaFuncSetAttribute(encode_kernel_static, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        int sms = 0, per_sm = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (e != cudaSuccess) return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, encode_kernel_static, kThreads,
                                                          smem);
        if (e != cudaSuccess) return e;
        s.grid = static_cast<uint32_t>(sms * (per_sm > 0 ? per_sm : 1));
        s.scratch = static_cast<uint64_t *>(address);
    }
    out = s;
    return cudaSuccess;
}

} // namespace
} // namespace tsk

extern "C" uint64_t tsk_encode_static_max_tiles(void) {
    return tsk::kStaticStateWords - 2;
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
    // The array keeps the previous call's contents: clear the counter and this call's flags.
    e = cudaMemsetAsync(setup.scratch, 0, tsk_encode_state_bytes(total), stream);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(result, 0, sizeof(tsk_result), stream);
    if (e != cudaSuccess) return e;
    const uint64_t grid = setup.grid < total ? setup.grid : total;
    tsk::encode_kernel_static<<<static_cast<uint32_t>(grid), tsk::kThreads,
                                sizeof(tsk::EncodeShared), stream>>>(*image, total, setup.scratch,
                                                                     result);
    return cudaGetLastError();
}
