// Staging the tiles of an ROI straight from an archive outside the GPU
// (include/tilestream/staging.h). A copy is a run of adjacent payloads (for a parsed file, one
// tile row of the ROI). When the archive is addressable from the device (pinned host memory,
// device memory) and every run is 4-byte aligned, the copies are made by one small kernel
// (kernels/stage.cu) per 160 runs; otherwise by one cudaMemcpyAsync per run.
#include <tilestream/staging.h>

#include "plan.h"

#include <vector>

namespace tilestream::cuda {
namespace {

// The ROI's tile rows [r0, r1] and columns [c0, c1] (the reference's intersecting tiles,
// tests/cuda_decoder_test.cpp:19-31, plan.cpp:281-349).
struct Span {
    std::uint64_t across = 0;
    std::uint64_t r0 = 0, r1 = 0, c0 = 0, c1 = 0;
};

Status span_of(const ImageMetadata &m, Roi roi, Span &s) noexcept {
    if (!host::supported_tile(m.tile) || m.image.width == 0 || m.image.height == 0) {
        return Status::invalid_argument;
    }
    s.across = host::ceil_div(m.image.width, m.tile.width);
    const std::uint64_t down = host::ceil_div(m.image.height, m.tile.height);
    if (m.tiles.size() != s.across * down) {
        return Status::invalid_argument;
    }
    if (roi.width == 0 || roi.height == 0 ||
        std::uint64_t{roi.x} + roi.width > m.image.width ||
        std::uint64_t{roi.y} + roi.height > m.image.height) {
        return Status::invalid_roi;
    }
    s.c0 = roi.x / m.tile.width;
    s.c1 = (std::uint64_t{roi.x} + roi.width - 1) / m.tile.width;
    s.r0 = roi.y / m.tile.height;
    s.r1 = (std::uint64_t{roi.y} + roi.height - 1) / m.tile.height;
    return Status::success;
}

// Calls copy(tiles, count, begin, end) for each copy, in file order: `count` tiles (their
// indices in tiles[0 .. count)) whose payloads lie one after another in file bytes
// [begin, end). The ROI's tiles are visited in row-major order, which for a parsed file is
// file order.
template <typename Copy> void for_each_copy(const ImageMetadata &m, const Span &s, Copy copy) {
    std::uint64_t tiles[512]; // the tiles of the copy being built (flushed when full)
    std::uint64_t count = 0, begin = 0, end = 0;
    for (std::uint64_t r = s.r0; r <= s.r1; ++r) {
        for (std::uint64_t c = s.c0; c <= s.c1; ++c) {
            const std::uint64_t t = r * s.across + c;
            const std::uint64_t a = m.tiles[t].offset, b = a + m.tiles[t].length;
            if (count != 0 && (a != end || count == 512)) {
                copy(tiles, count, begin, end);
                count = 0;
            }
            if (count == 0) {
                begin = a;
            }
            tiles[count++] = t;
            end = b;
        }
    }
    if (count != 0) {
        copy(tiles, count, begin, end);
    }
}

} // namespace

Status roi_staging_size(const ImageMetadata &metadata, Roi roi, RoiStaging &out) noexcept {
    Span s;
    const Status st = span_of(metadata, roi, s);
    if (st != Status::success) {
        return st;
    }
    RoiStaging r;
    for_each_copy(metadata, s,
                  [&](const std::uint64_t *, std::uint64_t count, std::uint64_t begin,
                      std::uint64_t end) {
                      r.tiles += count;
                      r.bytes += end - begin;
                      ++r.copies;
                  });
    out = r;
    return Status::success;
}

Status stage_roi_tiles(const ImageMetadata &metadata, Roi roi, ConstBytes archive,
                       MutableBytes staging, TileMapping *mappings,
                       std::uint64_t mapping_capacity, cudaStream_t stream,
                       RoiStaging &out) noexcept {
    if (archive.data == nullptr || staging.data == nullptr || mappings == nullptr ||
        archive.size < metadata.file_bytes) {
        return Status::invalid_argument;
    }
    RoiStaging need;
    Status st = roi_staging_size(metadata, roi, need);
    if (st != Status::success) {
        return st;
    }
    if (staging.size < need.bytes || mapping_capacity < need.tiles) {
        return Status::buffer_too_small;
    }
    Span s;
    static_cast<void>(span_of(metadata, roi, s));
    bool inside = true;
    for_each_copy(metadata, s,
                  [&](const std::uint64_t *, std::uint64_t, std::uint64_t begin,
                      std::uint64_t end) { inside = inside && begin <= end && end <= archive.size; });
    if (!inside) {
        return Status::invalid_argument;
    }
    int device = 0;
    st = detail::cuda_status(cudaGetDevice(&device), "cudaGetDevice");
    if (st != Status::success) {
        return st;
    }
    st = detail::stream_device(stream, device);
    if (st != Status::success) {
        return st;
    }
    st = detail::accessible(staging.data, device, false);
    if (st != Status::success) {
        return st;
    }
    // Where the device can read the archive, if it can: device memory of this device, managed
    // memory, or host memory that is pinned (and so mapped).
    const std::uint8_t *readable = nullptr;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, archive.data) == cudaSuccess) {
        if ((a.type == cudaMemoryTypeDevice && a.device == device) ||
            a.type == cudaMemoryTypeManaged) {
            readable = static_cast<const std::uint8_t *>(archive.data);
        } else if (a.type == cudaMemoryTypeHost && a.devicePointer != nullptr) {
            readable = static_cast<const std::uint8_t *>(a.devicePointer);
        }
    } else {
        static_cast<void>(cudaGetLastError());
    }
    struct Run {
        std::uint64_t begin, bytes, at;
    };
    std::vector<Run> runs;
    try {
        runs.reserve(static_cast<std::size_t>(need.copies));
    } catch (...) {
        return Status::resource_limit;
    }
    const auto *src = static_cast<const std::uint8_t *>(archive.data);
    auto *dst = static_cast<std::uint8_t *>(staging.data);
    std::uint64_t at = 0, k = 0;
    bool words = readable != nullptr && (reinterpret_cast<std::uintptr_t>(readable) % 4) == 0 &&
                 (reinterpret_cast<std::uintptr_t>(dst) % 4) == 0;
    for_each_copy(metadata, s,
                  [&](const std::uint64_t *tiles, std::uint64_t count, std::uint64_t begin,
                      std::uint64_t end) {
                      for (std::uint64_t i = 0; i < count; ++i) {
                          mappings[k++] = {tiles[i], at + (metadata.tiles[tiles[i]].offset - begin)};
                      }
                      const std::uint64_t bytes = end - begin;
                      words = words && begin % 4 == 0 && bytes % 4 == 0 && at % 4 == 0 &&
                              bytes < (1ull << 31);
                      runs.push_back({begin, bytes, at});
                      at += bytes;
                  });
    cudaError_t e = cudaSuccess;
    if (words) {
        tsk_stage_batch batch{};
        for (std::size_t i = 0; i < runs.size() && e == cudaSuccess; ++i) {
            tsk_stage_run &r = batch.runs[batch.count++];
            r.src = reinterpret_cast<std::uint64_t>(readable + runs[i].begin);
            r.dst = reinterpret_cast<std::uint64_t>(dst + runs[i].at);
            r.bytes = static_cast<std::uint32_t>(runs[i].bytes);
            r.first_piece = batch.pieces;
            batch.pieces += static_cast<std::uint32_t>((runs[i].bytes + 4095) / 4096);
            if (batch.count == TSK_STAGE_MAX_RUNS || i + 1 == runs.size()) {
                e = static_cast<cudaError_t>(tsk_stage_launch(&batch, stream));
                batch = tsk_stage_batch{};
            }
        }
    } else {
        for (const Run &r : runs) {
            if (e == cudaSuccess) {
                e = cudaMemcpyAsync(dst + r.at, src + r.begin, static_cast<std::size_t>(r.bytes),
                                    cudaMemcpyDefault, stream);
            }
        }
    }
    if (e != cudaSuccess) {
        return detail::cuda_failure("ROI staging copies", e);
    }
    out = need;
    return Status::success;
}

} // namespace tilestream::cuda
