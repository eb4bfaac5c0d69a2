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
            for (x = threadIdx.x * 4; x < vec_end; x += kThreads * 4) {
                uint32_t v[4];
                if constexpr (F32) {
                    const uint4 q = __ldg(reinterpret_cast<const uint4 *>(in + 4ull * x));
                    v[0] = q.x, v[1] = q.y, v[2] = q.z, v[3] = q.w;
                } else {
                    const uint2 q = __ldg(reinterpret_cast<const uint2 *>(in + 2ull * x));
                    v[0] = q.x & 0xffffu, v[1] = q.x >> 16, v[2] = q.y & 0xffffu, v[3] = q.y >> 16;
                }
                float4 o = make_float4(im.offset, im.offset, im.offset, im.offset);
                float4 g = make_float4(im.gain, im.gain, im.gain, im.gain);
                if (om) o = __ldg(reinterpret_cast<const float4 *>(om + x));
                if (gm) g = __ldg(reinterpret_cast<const float4 *>(gm + x));
                float4 r;
                r.x = cal(to_float<F32>(v[0]), o.x, g.x);
                r.y = cal(to_float<F32>(v[1]), o.y, g.y);
                r.z = cal(to_float<F32>(v[2]), o.z, g.z);
                r.w = cal(to_float<F32>(v[3]), o.w, g.w);
                __stcs(reinterpret_cast<float4 *>(out + x), r);
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
