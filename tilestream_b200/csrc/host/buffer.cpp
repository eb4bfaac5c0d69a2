// DeviceBuffer and synchronize of include/tilestream/cuda.h.
//
// Contract (docs/api.md "Device buffers", "Batch plans and ownership"): memory comes from the
// stream-ordered allocator of the stream's device and is 256-byte aligned (workspace_alignment);
// a successful allocate() hands the previous memory back in the order of that stream; the
// destructor and move assignment hand memory back on cudaStreamPerThread without waiting.
#include "plan.h"

namespace tilestream::cuda {
namespace {

// Returns `p` to the stream-ordered allocator after the work already queued on `stream`.
Status give_back(void *p, cudaStream_t stream) noexcept {
    return p == nullptr ? Status::success
                        : detail::cuda_status(cudaFreeAsync(p, stream), "cudaFreeAsync");
}

} // namespace

DeviceBuffer::~DeviceBuffer() {
    static_cast<void>(give_back(data_, cudaStreamPerThread));
}

DeviceBuffer::DeviceBuffer(DeviceBuffer &&other) noexcept : data_(other.data_), size_(other.size_) {
    other.data_ = nullptr;
    other.size_ = 0;
}

DeviceBuffer &DeviceBuffer::operator=(DeviceBuffer &&other) noexcept {
    if (&other == this) {
        return *this;
    }
    void *const held = data_;
    data_ = other.data_;
    size_ = other.size_;
    other.data_ = nullptr;
    other.size_ = 0;
    static_cast<void>(give_back(held, cudaStreamPerThread));
    return *this;
}

Status DeviceBuffer::allocate(std::uint64_t bytes, cudaStream_t stream,
                              DeviceBuffer &buffer) noexcept {
    if (bytes > max_bytes) {
        return Status::size_overflow;
    }
    // A zero-byte request leaves `buffer` empty; otherwise the new block must be in hand (and
    // aligned) before the old one is given back, so a failure leaves `buffer` as it was.
    void *block = nullptr;
    if (bytes != 0) {
        const cudaError_t e = cudaMallocAsync(&block, static_cast<std::size_t>(bytes), stream);
        if (e != cudaSuccess) {
            return detail::cuda_status(e, "cudaMallocAsync");
        }
        if (reinterpret_cast<std::uintptr_t>(block) % workspace_alignment != 0) {
            static_cast<void>(give_back(block, stream));
            return Status::cuda_error;
        }
    }
    const Status returned = buffer.release(stream);
    buffer.data_ = block;
    buffer.size_ = block != nullptr ? bytes : 0;
    return returned;
}

Status DeviceBuffer::release(cudaStream_t stream) noexcept {
    void *const held = data_;
    data_ = nullptr;
    size_ = 0;
    return give_back(held, stream);
}

Status synchronize(cudaStream_t stream) noexcept {
    return detail::cuda_status(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
}

} // namespace tilestream::cuda
