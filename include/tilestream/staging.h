#pragma once
// Staging the tiles of an ROI from an archive outside the GPU. This is an extension; the
// reference API has no counterpart. Its benchmark gathers the intersecting tiles of each ROI
// with host copies into a second pinned buffer and copies that buffer to the device
// (benchmarks/codec_benchmark.cpp:153-320). Here the copies go straight from the archive: the
// ROI's tiles of one tile row are adjacent in a .tsc file (payloads follow the index order), so
// one copy per tile row moves them, with no host gather. When the archive is pinned host memory
// or device memory, one small kernel makes all the copies of a call (it reads the archive
// through its device address), so a call costs one launch of host time however many rows the
// ROI spans; a pageable archive takes one cudaMemcpyAsync per row.
#include <tilestream/cuda.h>

#include <cstdint>

namespace tilestream::cuda {

struct RoiStaging {
    std::uint64_t tiles = 0;  // tiles that intersect the ROI
    std::uint64_t bytes = 0;  // their payload bytes: the staging buffer needs this many
    std::uint64_t copies = 0; // runs of adjacent payloads (for a parsed file, at most one
                              // per tile row of the ROI)
};

// The tiles, bytes and copies of staging `roi` of the archive described by `metadata`.
// invalid_roi for an empty ROI or one outside the image; invalid_argument for metadata whose
// tile table does not match its image and tile shape.
Status roi_staging_size(const ImageMetadata &metadata, Roi roi, RoiStaging &out) noexcept;

// Enqueues on `stream` the copies that bring the payloads of the tiles intersecting `roi`
// from `archive` (the complete .tsc file, usually in pinned host memory; device memory works
// too) into `staging` (device memory of the stream's device), packed in tile order, and writes
// one TileMapping per tile (its index and its offset in `staging`, in tile order). Together
// with `metadata` they form the CompressedInput of a decode_roi or decode_calibrate item for
// `roi` whose plan runs on a stream ordered after these copies. The archive and the staging
// buffer must stay untouched until the copies have completed. Every check runs before the
// first copy is enqueued: buffer_too_small when `staging` or `mapping_capacity` is short,
// invalid_argument for null pointers, an archive shorter than the metadata's file, staging that
// is not device memory of the stream's device, or a tile outside the archive.
Status stage_roi_tiles(const ImageMetadata &metadata, Roi roi, ConstBytes archive,
                       MutableBytes staging, TileMapping *mappings,
                       std::uint64_t mapping_capacity, cudaStream_t stream,
                       RoiStaging &out) noexcept;

} // namespace tilestream::cuda
