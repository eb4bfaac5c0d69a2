// Standalone calibration y = RN(RN(x - offset) * gain) for sm_100a.
//
// The reference runs one warp per row of the concatenated batch with scalar 4-byte accesses and
// a binary search for the owning image (src/cuda/calibrate.cu:13-42), then a separate `report`
// kernel. Here the planner cuts the batch into row chunks of one image each; a persistent grid
// streams them with 16-byte loads and stores whenever the rows are aligned, and the first chunk
// of each image writes its DeviceResult. The arithmetic is the same as the fused decoder's
// (__fsub_rn then __fmul_rn, never contracted; no flush of subnormals), so fused and separate
// calibration give identical bits on one device.
#include "tasks.h"

#include <cstdint>

namespace tsk {
namespace {

constexpr uint32_t kThreads = 256;

__device__ __forceinline__ float cal(float x, float o, float g) {
    return __fmul_rn(__fsub_rn(x, o), g);
}

template <bool F32> __device__ __forceinline__ float to_float(uint32_t v) {
    if constexpr (F32) {
        return __uint_as_float(v);
    } else {
        return static_cast<float>(v);
    }
}

template <bool F32>
__device__ void calibrate_rows(const tsk_calib_image &im, uint32_t y0, uint32_t rows) {
    constexpr uint32_t s = F32 ? 4 : 2;
    const uint32_t width = im.width;
    for (uint32_t y = y0; y < y0 + rows; ++y) {
        const uint8_t *in = reinterpret_cast<const uint8_t *>(im.input) + y * im.in_pitch;
        float *out = reinterpret_cast<float *>(im.out + y * im.out_pitch);
        const float *om =
            im.offset_map ? reinterpret_cast<const float *>(im.offset_map + y * im.offset_pitch)
                          : nullptr;
        const float *gm =
            im.gain_map ? reinterpret_cast<const float *>(im.gain_map + y * im.gain_pitch)
                        : nullptr;
        const uintptr_t misalign = (reinterpret_cast<uintptr_t>(in) % (4 * s)) |
                                   (reinterpret_cast<uintptr_t>(out) % 16) |
                                   (reinterpret_cast<uintptr_t>(om) % 16) |
                                   (reinterpret_cast<uintptr_t>(gm) % 16);
        uint32_t x = 0;
        if (misalign == 0) {
            const uint32_t vec_end = width & ~3u;
            constexpr uint32_t kStep = kThreads * 4;
            // Groups of four samples; two groups per iteration, all their loads issued before
            // any result is computed.
            struct Group {
                uint32_t v[4];
                float4 o, g;
            };
            auto load = [&](uint32_t at, Group &q) {
                if constexpr (F32) {
                    const uint4 w = __ldg(reinterpret_cast<const uint4 *>(in + 4ull * at));
                    q.v[0] = w.x, q.v[1] = w.y, q.v[2] = w.z, q.v[3] = w.w;
                } else {
                    const uint2 w = __ldg(reinterpret_cast<const uint2 *>(in + 2ull * at));
                    q.v[0] = w.x & 0xffffu, q.v[1] = w.x >> 16;
                    q.v[2] = w.y & 0xffffu, q.v[3] = w.y >> 16;
                }
                q.o = om ? __ldg(reinterpret_cast<const float4 *>(om + at))
                         : make_float4(im.offset, im.offset, im.offset, im.offset);
                q.g = gm ? __ldg(reinterpret_cast<const float4 *>(gm + at))
                         : make_float4(im.gain, im.gain, im.gain, im.gain);
            };
            auto store = [&](uint32_t at, const Group &q) {
                float4 r;
                r.x = cal(to_float<F32>(q.v[0]), q.o.x, q.g.x);
                r.y = cal(to_float<F32>(q.v[1]), q.o.y, q.g.y);
                r.z = cal(to_float<F32>(q.v[2]), q.o.z, q.g.z);
                r.w = cal(to_float<F32>(q.v[3]), q.o.w, q.g.w);
                __stcs(reinterpret_cast<float4 *>(out + at), r);
            };
            for (x = threadIdx.x * 4; x + kStep < vec_end; x += 2 * kStep) {
                Group a, b;
                load(x, a);
                load(x + kStep, b);
                store(x, a);
                store(x + kStep, b);
            }
            if (x < vec_end) {
                Group a;
                load(x, a);
                store(x, a);
            }
            x = vec_end + threadIdx.x;
        } else {
            x = threadIdx.x;
        }
        for (; x < width; x += kThreads) {
            uint32_t v;
            if constexpr (F32) {
                v = reinterpret_cast<const uint32_t *>(in)[x];
            } else {
                v = reinterpret_cast<const uint16_t *>(in)[x];
            }
            out[x] = cal(to_float<F32>(v), om ? om[x] : im.offset, gm ? gm[x] : im.gain);
        }
    }
}

__global__ void __launch_bounds__(kThreads)
    calibrate_kernel(const tsk_calib_task *__restrict__ tasks, uint32_t ntasks,
                     const tsk_calib_image *__restrict__ images, tsk_result *results) {
    for (uint32_t i = blockIdx.x; i < ntasks; i += gridDim.x) {
        const tsk_calib_task t = tasks[i];
        const tsk_calib_image &im = images[t.image];
        if (im.type == 2) {
            calibrate_rows<true>(im, t.y0, t.rows);
        } else {
            calibrate_rows<false>(im, t.y0, t.rows);
        }
        if (t.reserved != 0 && threadIdx.x == 0) {
            tsk_result r;
            r.status = 0;
            r.reserved = 0;
            r.bytes_written = 4ull * im.width * im.height;
            results[t.image] = r;
        }
    }
}

} // namespace
} // namespace tsk

extern "C" int tsk_calibrate_prepare(int device) {
    (void)device;
    cudaFuncAttributes attributes;
    return cudaFuncGetAttributes(&attributes, tsk::calibrate_kernel);
}

extern "C" int tsk_calibrate_launch(const tsk_calib_task *tasks, uint32_t ntasks,
                                    const tsk_calib_image *images, uint32_t image_count,
                                    tsk_result *results, cudaStream_t stream) {
    (void)image_count;
    if (ntasks == 0) return cudaSuccess;
    int device = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tsk::calibrate_kernel,
                                                      tsk::kThreads, 0);
    if (e != cudaSuccess) return e;
    uint64_t grid = static_cast<uint64_t>(sms) * (per_sm > 0 ? per_sm : 1);
    if (grid > ntasks) grid = ntasks;
    tsk::calibrate_kernel<<<static_cast<uint32_t>(grid), tsk::kThreads, 0, stream>>>(
        tasks, ntasks, images, results);
    return cudaGetLastError();
}
