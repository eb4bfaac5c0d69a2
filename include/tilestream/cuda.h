#pragma once
// Drop-in replacement for the reference's include/tilestream/cuda.h (cuda.h:1-191): CUDA plan
// preparation and the five asynchronous executors. Every declaration and record layout matches
// the reference (DeviceSegment 16 B, DeviceTile 40 B, DeviceResult 16 B); the plan internals
// behind BatchPlan::Impl are this library's own.
#include <tilestream/build_config.h>

#if TILESTREAM_WITH_CUDA

#include <tilestream/api.h>

#include <cuda_runtime_api.h>

#include <cstdint>
#include <memory>

namespace tilestream::cuda {

enum class Operation : std::uint32_t {
    compress,
    decompress,
    decode_roi,
    calibrate,
    decode_calibrate,
};

enum class ParameterKind : std::uint32_t { scalar, map };

// A calibration parameter: one value, or an FP32 map in output-region coordinates.
struct Parameter {
    ParameterKind kind = ParameterKind::scalar;
    float scalar = 0.0F;
    ConstImageView map;
};

// y = (x - offset) * gain, rounded after the subtraction and after the multiplication.
struct Calibration {
    Parameter offset;
    Parameter gain{ParameterKind::scalar, 1.0F, {}};
};

// A staged payload: tile tile_index of the archive lives at input_offset in the device bytes.
struct TileMapping {
    std::uint64_t tile_index = 0;
    std::uint64_t input_offset = 0;
};

struct CompressedInput {
    ConstBytes bytes;
    const ImageMetadata *metadata = nullptr;
    const TileMapping *mappings = nullptr;
    std::uint64_t mapping_count = 0;
    // Trusted path: bytes are the output of this library's encoder, described by its result.
    const DeviceResult *encoder_result = nullptr;
    ImageSpec trusted_image;
    TileShape trusted_tile;
};

struct BatchItem {
    ConstImageView input;
    ImageView output;
    MutableBytes compressed_output;
    CompressedInput compressed_input;
    Roi roi;
    Calibration calibration;
};

struct BatchRequest {
    Operation operation = Operation::compress;
    const BatchItem *items = nullptr;
    std::uint64_t count = 0;
    TileShape tile;
};

// Native device records of the reference API. They are part of the public ABI; this
// implementation plans with its own task records and keeps these for source compatibility.
struct DeviceSegment {
    std::uint32_t seed = 0;
    std::uint32_t bit_width = 0;
    std::uint64_t input_offset = 0;
};

struct DeviceTile {
    std::uint64_t tile_index = 0;
    std::uint64_t input_offset = 0;
    std::uint64_t length = 0;
    std::uint64_t first_segment = 0;
    TileMode mode = TileMode::raw;
    std::uint16_t width = 0;
    std::uint16_t height = 0;
};

struct DeviceImage {
    ConstImageView input;
    ImageView output;
    ConstBytes compressed_input;
    MutableBytes compressed_output;
    const DeviceTile *tiles = nullptr;
    const DeviceSegment *segments = nullptr;
    std::uint64_t tile_count = 0;
    const DeviceResult *encoder_result = nullptr;
    ImageSpec archive_image;
    TileShape archive_tile;
    Roi roi;
    Calibration calibration;
};

struct DeviceBatch {
    const DeviceImage *images = nullptr;
    std::uint32_t count = 0;
};

struct ResultBuffer {
    DeviceResult *data = nullptr;
    std::uint64_t count = 0;
};

// Device memory from the stream-ordered allocator, aligned to workspace_alignment. Execution
// functions never allocate; this is a convenience for callers.
class DeviceBuffer {
  public:
    DeviceBuffer() noexcept = default;
    // Frees on cudaStreamPerThread without waiting: all work using the memory must be done.
    ~DeviceBuffer();
    DeviceBuffer(DeviceBuffer &&other) noexcept;
    DeviceBuffer &operator=(DeviceBuffer &&other) noexcept;
    DeviceBuffer(const DeviceBuffer &) = delete;
    DeviceBuffer &operator=(const DeviceBuffer &) = delete;

    // On success the buffer's previous memory is freed in stream order.
    [[nodiscard]] static Status allocate(std::uint64_t bytes, cudaStream_t stream,
                                         DeviceBuffer &buffer) noexcept;
    // Frees after the work already enqueued in stream.
    [[nodiscard]] Status release(cudaStream_t stream) noexcept;

    [[nodiscard]] void *data() const noexcept {
        return data_;
    }
    [[nodiscard]] std::uint64_t size() const noexcept {
        return size_;
    }
    [[nodiscard]] MutableBytes bytes() const noexcept {
        return {data_, size_};
    }

  private:
    void *data_ = nullptr;
    std::uint64_t size_ = 0;
};

// Waits for stream; any launch or execution failure seen there is cuda_error.
[[nodiscard]] Status synchronize(cudaStream_t stream) noexcept;

// One execution at a time per plan; concurrent executions need separate plans.
class BatchPlan {
  public:
    ~BatchPlan();
    BatchPlan(const BatchPlan &) = delete;
    BatchPlan &operator=(const BatchPlan &) = delete;
    BatchPlan(BatchPlan &&) noexcept;
    BatchPlan &operator=(BatchPlan &&) noexcept;

    [[nodiscard]] WorkspaceSpec workspace_spec() const noexcept;

  private:
    struct Impl;
    std::unique_ptr<Impl> impl_;
    explicit BatchPlan(std::unique_ptr<Impl> impl) noexcept;
    friend Status prepare_batch(const BatchRequest &, std::unique_ptr<BatchPlan> &,
                                cudaStream_t) noexcept;
    friend Status compress_async(const BatchPlan &, MutableBytes, ResultBuffer,
                                 cudaStream_t) noexcept;
    friend Status decompress_async(const BatchPlan &, MutableBytes, ResultBuffer,
                                   cudaStream_t) noexcept;
    friend Status decode_roi_async(const BatchPlan &, MutableBytes, ResultBuffer,
                                   cudaStream_t) noexcept;
    friend Status calibrate_async(const BatchPlan &, MutableBytes, ResultBuffer,
                                  cudaStream_t) noexcept;
    friend Status decode_calibrate_async(const BatchPlan &, MutableBytes, ResultBuffer,
                                         cudaStream_t) noexcept;
    friend struct PlanAccess;
};

[[nodiscard]] Status prepare_batch(const BatchRequest &request, std::unique_ptr<BatchPlan> &plan,
                                   cudaStream_t stream) noexcept;
[[nodiscard]] Status compress_async(const BatchPlan &plan, MutableBytes workspace,
                                    ResultBuffer results, cudaStream_t stream) noexcept;
[[nodiscard]] Status decompress_async(const BatchPlan &plan, MutableBytes workspace,
                                      ResultBuffer results, cudaStream_t stream) noexcept;
[[nodiscard]] Status decode_roi_async(const BatchPlan &plan, MutableBytes workspace,
                                      ResultBuffer results, cudaStream_t stream) noexcept;
[[nodiscard]] Status calibrate_async(const BatchPlan &plan, MutableBytes workspace,
                                     ResultBuffer results, cudaStream_t stream) noexcept;
[[nodiscard]] Status decode_calibrate_async(const BatchPlan &plan, MutableBytes workspace,
                                            ResultBuffer results, cudaStream_t stream) noexcept;

} // namespace tilestream::cuda

#endif
