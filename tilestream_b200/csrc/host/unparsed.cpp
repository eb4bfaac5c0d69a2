// Whole-image decode of files never parsed on the host (include/tilestream/unparsed.h).
//
// The host checks each file's header (the parser's header rules, from the caller's host copy),
// the arguments and the aliasing rule, and fills one launch record per file; the decoder derives
// one task per tile from the record (FileSource in kernels/decode.cu) and validates the index
// entries, payloads and row descriptors on the device.
#include <tilestream/unparsed.h>

#include "../kernels/tasks.h"
#include "plan.h"

#include <cstring>

namespace tilestream::cuda {

Status decode_unparsed_async(const UnparsedFile *files, std::uint64_t count, ResultBuffer results,
                             cudaStream_t stream) noexcept {
    if (count == 0) {
        return Status::success;
    }
    if (files == nullptr || results.data == nullptr) {
        return Status::invalid_argument;
    }
    if (count > max_unparsed_files) {
        return Status::resource_limit;
    }
    if (results.count < count) {
        return Status::buffer_too_small;
    }
    if (reinterpret_cast<std::uintptr_t>(results.data) % alignof(DeviceResult) != 0) {
        return Status::invalid_argument;
    }
    static_assert(max_unparsed_files == TSK_FILE_MAX_BATCH, "one launch record per file");
    const std::uint64_t record_bytes = count * sizeof(DeviceResult);
    for (std::uint64_t j = 0; j < count; ++j) {
        if (host::overlaps(results.data, record_bytes, files[j].bytes.data, files[j].bytes.size)) {
            return Status::invalid_argument;
        }
    }
    tsk_file_batch batch{};
    bool any_f32 = false;
    std::uint64_t ntasks = 0;
    for (std::uint64_t i = 0; i < count; ++i) {
        const UnparsedFile &f = files[i];
        if (f.header == nullptr) {
            return Status::invalid_argument;
        }
        Status st = host::byte_range(f.bytes.data, f.bytes.size);
        if (st != Status::success) {
            return st;
        }
        if (f.bytes.data == nullptr || reinterpret_cast<std::uintptr_t>(f.bytes.data) % 4 != 0) {
            return Status::invalid_argument;
        }
        ImageSpec image{};
        TileShape tile{};
        std::uint64_t tiles = 0;
        st = host::check_file_header(static_cast<const std::uint8_t *>(f.header), f.bytes.size,
                                     image, tile, tiles);
        if (st != Status::success) {
            return st;
        }
        st = host::view_ok(f.output);
        if (st != Status::success) {
            return st;
        }
        if (f.output.image.type != image.type || f.output.image.width != image.width ||
            f.output.image.height != image.height) {
            return Status::invalid_argument;
        }
        // Outputs are written: they may overlap no input, no other output and no record.
        if (host::overlaps(f.output.data, f.output.capacity_bytes, results.data, record_bytes)) {
            return Status::invalid_argument;
        }
        for (std::uint64_t j = 0; j < count; ++j) {
            if (host::overlaps(f.output.data, f.output.capacity_bytes, files[j].bytes.data,
                               files[j].bytes.size) ||
                (j != i && host::overlaps(f.output.data, f.output.capacity_bytes,
                                          files[j].output.data, files[j].output.capacity_bytes))) {
                return Status::invalid_argument;
            }
        }
        ntasks += tiles;
        if (ntasks > UINT32_MAX) {
            return Status::resource_limit;
        }
        const bool f32 = image.type == PixelType::float32;
        any_f32 = any_f32 || f32;
        tsk_file &rec = batch.files[i];
        rec.image.out = reinterpret_cast<std::uint64_t>(f.output.data);
        rec.image.out_pitch = f.output.pitch_bytes;
        rec.image.gain = 1.0f;
        rec.image.result_bytes = std::uint64_t{image.width} * image.height * (f32 ? 4 : 2);
        rec.image.capacity = f.bytes.size;
        rec.image.tile_count = static_cast<std::uint32_t>(tiles);
        rec.image.archive_width = image.width;
        rec.image.archive_height = image.height;
        rec.image.tile_width = tile.width;
        rec.image.tile_height = tile.height;
        rec.src = reinterpret_cast<std::uint64_t>(f.bytes.data);
        rec.task_end = static_cast<std::uint32_t>(ntasks);
        rec.tiles_across = static_cast<std::uint32_t>(host::ceil_div(image.width, tile.width));
        rec.flags = f32 ? TSK_F32 : 0;
        std::memcpy(rec.header, f.header, sizeof(rec.header));
    }
    batch.count = static_cast<std::uint32_t>(count);
    batch.ntasks = static_cast<std::uint32_t>(ntasks);

    int device = 0, pageable = 0;
    if (cudaGetDevice(&device) != cudaSuccess ||
        cudaDeviceGetAttribute(&pageable, cudaDevAttrPageableMemoryAccess, device) != cudaSuccess) {
        return detail::cuda_failure("cudaGetDevice/cudaDeviceGetAttribute");
    }
    Status st = detail::stream_device(stream, device);
    for (std::uint64_t i = 0; i < count && st == Status::success; ++i) {
        st = detail::accessible(files[i].bytes.data, device, pageable != 0);
        if (st == Status::success) {
            st = detail::accessible(files[i].output.data, device, pageable != 0);
        }
    }
    if (st == Status::success) {
        st = detail::accessible(results.data, device, pageable != 0);
    }
    if (st == Status::success) {
        const cudaError_t pending = cudaPeekAtLastError();
        if (pending != cudaSuccess) {
            detail::log_failure("pending error before enqueue (left for the caller)", pending);
            st = Status::cuda_error;
        }
    }
    if (st != Status::success) {
        return st;
    }
    std::uint32_t grid = 0;
    const int e = tsk_file_prepare(any_f32 ? 1 : 0, device, &grid);
    if (e != 0) {
        return detail::cuda_failure("unparsed-file kernel preload", static_cast<cudaError_t>(e));
    }
    return detail::cuda_status(tsk_file_launch(&batch, reinterpret_cast<tsk_result *>(results.data),
                                               grid, any_f32 ? 1 : 0, stream),
                               "unparsed-file decode launch");
}

} // namespace tilestream::cuda
