// Staging copies of an ROI's tile payloads (host side: csrc/host/staging.cpp) as one small
// kernel: each CTA copies 4 KiB pieces of the runs, reading the archive through its device
// address (pinned host memory over the host link, or device memory) with 4-byte loads, several
// in flight per thread. One launch replaces one cudaMemcpyAsync per run, whose host cost
// (a few microseconds each) bounds a pipeline of small ROIs.
#include "tasks.h"

#include <cstdint>

namespace tsk {
namespace {

constexpr uint32_t kThreads = 256;
constexpr uint32_t kPieceBytes = 4096;
constexpr uint32_t kWordsPerThread = kPieceBytes / 4 / kThreads; // 4

__global__ void __launch_bounds__(kThreads)
    stage_kernel(const __grid_constant__ tsk_stage_batch batch) {
    for (uint32_t p = blockIdx.x; p < batch.pieces; p += gridDim.x) {
        // The run holding piece p: the last one whose first piece is at or before p.
        uint32_t lo = 0, hi = batch.count;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) / 2;
            if (batch.runs[mid].first_piece <= p) {
                lo = mid;
            } else {
                hi = mid;
            }
        }
        const tsk_stage_run &run = batch.runs[lo];
        const uint32_t off = (p - run.first_piece) * kPieceBytes;
        const uint32_t words = (run.bytes - off < kPieceBytes ? run.bytes - off : kPieceBytes) / 4;
        const uint32_t *src = reinterpret_cast<const uint32_t *>(run.src + off);
        uint32_t *dst = reinterpret_cast<uint32_t *>(run.dst + off);
        uint32_t v[kWordsPerThread];
#pragma unroll
        for (uint32_t k = 0; k < kWordsPerThread; ++k) {
            const uint32_t i = threadIdx.x + k * kThreads;
            v[k] = i < words ? src[i] : 0u;
        }
#pragma unroll
        for (uint32_t k = 0; k < kWordsPerThread; ++k) {
            const uint32_t i = threadIdx.x + k * kThreads;
            if (i < words) {
                dst[i] = v[k];
            }
        }
    }
}

} // namespace
} // namespace tsk

extern "C" int tsk_stage_launch(const tsk_stage_batch *batch, cudaStream_t stream) {
    if (batch->pieces == 0) return cudaSuccess;
    const uint32_t grid = batch->pieces < 592 ? batch->pieces : 592;
    tsk::stage_kernel<<<grid, tsk::kThreads, 0, stream>>>(*batch);
    return cudaGetLastError();
}
