// Internal plan state behind tilestream::cuda::BatchPlan.
#pragma once

#include <tilestream/cuda.h>

#include "../kernels/tasks.h"
#include "checked.h"

#include <cstdint>
#include <vector>

namespace tilestream::cuda::detail {

struct Range {
    std::uintptr_t begin = 0;
    std::uintptr_t end = 0;
};

// The byte ranges one plan touches. Writable ranges may overlap nothing else; readable ranges
// may overlap one another (docs/api.md "Aliasing"). After a successful assign() the set keeps
// only the union of all its ranges, coalesced into sorted disjoint spans, which is what an
// execution's workspace and result records are checked against.
class RangeSet {
  public:
    // False when a writable range overlaps any other range of either kind.
    [[nodiscard]] bool assign(std::vector<Range> writable, std::vector<Range> readable);
    // True when `range` shares no byte with any range of the set (empty ranges share none).
    [[nodiscard]] bool disjoint(Range range) const noexcept;

  private:
    std::vector<Range> spans_; // sorted by begin, pairwise disjoint and non-adjacent
};

inline Range range_of(const void *data, std::uint64_t size) noexcept {
    const auto b = reinterpret_cast<std::uintptr_t>(data);
    return {b, b + static_cast<std::uintptr_t>(size)};
}

// Writes "tilestream: <what> failed: <error>" to stderr when TILESTREAM_DEBUG is set.
void log_failure(const char *what, cudaError_t error) noexcept;

// A CUDA failure is reported through Status; the error is cleared so a later check cannot
// blame it on another launch (reference plan.h:84-91).
inline Status cuda_failure(const char *what = "CUDA runtime call",
                           cudaError_t error = cudaErrorUnknown) noexcept {
    const cudaError_t last = cudaGetLastError();
    log_failure(what, error != cudaErrorUnknown ? error : last);
    return Status::cuda_error;
}

inline Status cuda_status(cudaError_t e, const char *what = "CUDA runtime call") noexcept {
    return e == cudaSuccess ? Status::success : cuda_failure(what, e);
}

inline Status cuda_status(int e, const char *what = "CUDA runtime call") noexcept {
    return cuda_status(static_cast<cudaError_t>(e), what);
}

[[nodiscard]] Status accessible(const void *data, int device, bool pageable) noexcept;
[[nodiscard]] Status stream_device(cudaStream_t stream, int device) noexcept;

struct PlanState {
    Operation operation = Operation::compress;
    PixelType type = PixelType::uint16;
    int device = 0;
    bool pageable = false;
    std::uint64_t count = 0;
    WorkspaceSpec spec;
    host::WorkspaceLayout layout;
    RangeSet ranges;
    void *storage = nullptr; // one device allocation holding every table

    // Decode.
    const tsk_decode_task *tasks = nullptr;
    std::uint32_t task_count = 0;
    const tsk_decode_image *images = nullptr;
    const tsk_row_start *rows = nullptr;
    tsk_decode_config config{};
    std::uint32_t *claims = nullptr; // the work queue's counter (dynamic kernel shapes)
    bool trusted = false;

    // Encode.
    const tsk_encode_image *encode_images = nullptr;
    std::uint64_t total_tiles = 0;

    // Standalone calibration.
    const tsk_calib_task *calib_tasks = nullptr;
    std::uint32_t calib_task_count = 0;
    const tsk_calib_image *calib_images = nullptr;

    PlanState() = default;
    PlanState(const PlanState &) = delete;
    PlanState &operator=(const PlanState &) = delete;
    ~PlanState();
};

// The structural checks of tile `index` that keep device reads inside its payload.
[[nodiscard]] Status check_tile(const ImageMetadata &m, std::uint64_t index) noexcept;

// One tile task of a decode plan as the host planned it (inspect_decode): the bytes it stages,
// the output bytes it may write, and for parsed predictive tiles the end of its furthest row
// descriptor relative to read_begin.
struct TaskSpan {
    std::uint64_t image = 0;
    std::uint64_t read_begin = 0, read_end = 0;
    std::uint64_t write_begin = 0, write_end = 0;
    std::uint64_t rows_end = 0;
    std::uint32_t mode = 0, flags = 0;
    std::uint32_t width = 0, height = 0;
};

[[nodiscard]] Status inspect_decode(const BatchRequest &request, std::vector<TaskSpan> &spans);

[[nodiscard]] Status check_execution(const PlanState *plan, Operation operation,
                                     MutableBytes workspace, ResultBuffer results,
                                     cudaStream_t stream) noexcept;

} // namespace tilestream::cuda::detail

namespace tilestream::cuda {

struct BatchPlan::Impl final : detail::PlanState {};

// Access to plan internals for the library's own extensions (C entry layer, batching).
struct PlanAccess {
    static const detail::PlanState *state(const BatchPlan &plan) noexcept {
        return plan.impl_.get();
    }
};

} // namespace tilestream::cuda
