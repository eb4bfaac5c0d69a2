// DeviceBuffer and synchronize of include/tilestream/cuda.h (reference: src/cuda/buffer.cpp).
#include "plan.h"

#include <utility>

namespace tilestream::cuda {

DeviceBuffer::~DeviceBuffer() {
    if (data_ != nullptr) {
        static_cast<void>(detail::cuda_status(cudaFreeAsync(data_, cudaStreamPerThread)));
    }
}

DeviceBuffer::DeviceBuffer(DeviceBuffer &&other) noexcept
    : data_(std::exchange(other.data_, nullptr)), size_(std::exchange(other.size_, 0)) {}

DeviceBuffer &DeviceBuffer::operator=(DeviceBuffer &&other) noexcept {
    if (this != &other) {
        DeviceBuffer previous(std::move(*this));
        data_ = std::exchange(other.data_, nullptr);
        size_ = std::exchange(other.size_, 0);
    }
    return *this;
}

Status DeviceBuffer::allocate(std::uint64_t bytes, cudaStream_t stream,
                              DeviceBuffer &buffer) noexcept {
    if (bytes > max_bytes) {
        return Status::size_overflow;
    }
    DeviceBuffer fresh;
    if (bytes != 0) {
        if (cudaMallocAsync(&fresh.data_, static_cast<std::size_t>(bytes), stream) != cudaSuccess) {
            fresh.data_ = nullptr;
            return detail::cuda_failure();
        }
        fresh.size_ = bytes;
        if (reinterpret_cast<std::uintptr_t>(fresh.data_) % workspace_alignment != 0) {
            static_cast<void>(fresh.release(stream));
            return Status::cuda_error;
        }
    }
    const Status st = buffer.release(stream);
    buffer = std::move(fresh);
    return st;
}

Status DeviceBuffer::release(cudaStream_t stream) noexcept {
    if (data_ == nullptr) {
        return Status::success;
    }
    const cudaError_t e = cudaFreeAsync(data_, stream);
    data_ = nullptr;
    size_ = 0;
    return detail::cuda_status(e);
}

Status synchronize(cudaStream_t stream) noexcept {
    return detail::cuda_status(cudaStreamSynchronize(stream));
}

} // namespace tilestream::cuda
