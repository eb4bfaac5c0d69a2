#pragma once
// Mixed batches: many archives and ROIs of uneven sizes, mixed pixel types, tile geometries and
// operations decoded by ONE persistent kernel from one device task queue, launched as a CUDA
// graph, with an optional autotuner. This is an extension; the reference API has no
// counterpart (one reference batch has one pixel type and one operation, see cuda.h).
#include <tilestream/cuda.h>

#include <cstdint>
#include <memory>

namespace tilestream::cuda {

// One decode of a mixed batch: an operation (decompress, decode_roi or decode_calibrate) and
// its item, with exactly the meaning and validation of that operation in prepare_batch.
struct MixedItem {
    Operation operation = Operation::decompress;
    BatchItem item;
};

struct MixedOptions {
    // Executions replay a CUDA graph instantiated by the preparation (one kernel node, plus a
    // clear of the result records when the batch has trusted encoder-output items).
    bool graph = true;
    // Chooses the kernel shape (consumer warps x columns per lane) and the persistent grid by
    // timing candidate configurations during the preparation. Tuning executes the batch, so
    // outputs and results are written. Choices are remembered per device and workload in the
    // process and, when tune_cache names a file, across processes.
    bool autotune = false;
    const char *tune_cache = nullptr;
    // A fixed kernel shape (0 .. decode_shape_count() - 1) instead of the default one, with the
    // occupancy-derived grid; the autotuner is then not run. -1: the default shape. Used to
    // check each shape's output and to measure shapes against each other.
    std::int32_t shape = -1;
};

// The number of kernel shapes a MixedOptions::shape may name.
[[nodiscard]] std::uint32_t decode_shape_count() noexcept;

struct MixedStats {
    std::uint64_t tiles = 0;  // tasks in the device queue
    std::uint32_t shape = 0;  // kernel shape
    std::uint32_t grid = 0;   // persistent CTAs
    std::uint32_t per_sm = 0; // resident CTAs per SM at that grid
    std::uint32_t graph = 0;  // 1 when executions replay a CUDA graph
    float tuned_us = 0.0f;    // time of the chosen configuration (0 when not tuned)
};

class MixedBatch {
  public:
    ~MixedBatch();
    MixedBatch(const MixedBatch &) = delete;
    MixedBatch &operator=(const MixedBatch &) = delete;
    struct Impl;

  private:
    std::unique_ptr<Impl> impl_;
    explicit MixedBatch(std::unique_ptr<Impl> impl) noexcept;
    friend struct MixedAccess;
};

// Validates every item as prepare_batch validates an item of its operation (statuses included),
// binds the result buffer (one record per item, in item order) and builds the task queue. The
// batch, like a plan, runs one execution at a time.
[[nodiscard]] Status prepare_mixed_batch(const MixedItem *items, std::uint64_t count,
                                         ResultBuffer results, const MixedOptions &options,
                                         std::unique_ptr<MixedBatch> &batch,
                                         cudaStream_t stream) noexcept;
// Enqueues one execution; asynchronous like the *_async executors.
[[nodiscard]] Status run_mixed_batch(const MixedBatch &batch, cudaStream_t stream) noexcept;
[[nodiscard]] MixedStats mixed_batch_stats(const MixedBatch &batch) noexcept;

} // namespace tilestream::cuda
