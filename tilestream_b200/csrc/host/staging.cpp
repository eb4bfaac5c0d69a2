// Staging the tiles of an ROI straight from an archive outside the GPU
// (include/tilestream/staging.h). Host code only: the copies are cudaMemcpyAsync calls, one per
// run of adjacent payloads (for a parsed file, one per tile row of the ROI), runs closer than
// 64 KiB being merged into one copy.
#include <tilestream/staging.h>

#include "plan.h"

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

// Bytes between two runs below which they are copied as one (the gap goes along): a copy
// costs a few microseconds of host time, in which the host link moves about 150 KB.
constexpr std::uint64_t kMergeGap = 64 * 1024;

// Calls copy(tiles, count, begin, end) for each copy, in file order: `count` tiles (their
// indices in tiles[0 .. count)) whose payloads lie in file bytes [begin, end). A copy is a run
// of tiles whose payloads follow one another, extended over gaps of at most kMergeGap bytes to
// the next run. The ROI's tiles are visited in row-major order, which for a parsed file is file
// order; tiles stored out of order start a new copy.
template <typename Copy> void for_each_copy(const ImageMetadata &m, const Span &s, Copy copy) {
    std::uint64_t tiles[512]; // the tiles of the copy being built (flushed when full)
    std::uint64_t count = 0, begin = 0, end = 0;
    for (std::uint64_t r = s.r0; r <= s.r1; ++r) {
        for (std::uint64_t c = s.c0; c <= s.c1; ++c) {
            const std::uint64_t t = r * s.across + c;
            const std::uint64_t a = m.tiles[t].offset, b = a + m.tiles[t].length;
            if (count != 0 && (a < end || a - end > kMergeGap || count == 512)) {
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
    const auto *src = static_cast<const std::uint8_t *>(archive.data);
    auto *dst = static_cast<std::uint8_t *>(staging.data);
    std::uint64_t at = 0, k = 0;
    cudaError_t e = cudaSuccess;
    for_each_copy(metadata, s,
                  [&](const std::uint64_t *tiles, std::uint64_t count, std::uint64_t begin,
                      std::uint64_t end) {
                      for (std::uint64_t i = 0; i < count; ++i) {
                          mappings[k++] = {tiles[i], at + (metadata.tiles[tiles[i]].offset - begin)};
                      }
                      if (e == cudaSuccess) {
                          e = cudaMemcpyAsync(dst + at, src + begin,
                                              static_cast<std::size_t>(end - begin),
                                              cudaMemcpyDefault, stream);
                      }
                      at += end - begin;
                  });
    if (e != cudaSuccess) {
        return detail::cuda_failure("cudaMemcpyAsync (ROI staging)", e);
    }
    out = need;
    return Status::success;
}

} // namespace tilestream::cuda
