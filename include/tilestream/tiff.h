// TIFF import and export of single-channel images (reference include/tilestream/tiff.h:10-37).
//
// The step before encode for real data: read_tiff loads one baseline TIFF image (uint16 or
// FP32 samples, one channel, strips or tiles, uncompressed or Deflate, optional predictor) into
// a packed host image; write_tiff stores an image as a tiled TIFF. The library reads and writes
// the TIFF container itself (no libtiff); Deflate streams go through zlib.
//
// read_tiff accepts: classic TIFF and BigTIFF, either byte order; exactly one image directory;
// SamplesPerPixel 1, PlanarConfiguration 1, Orientation 1 (top-left), Photometric 1
// (min-is-black; assumed when absent); BitsPerSample 16 with SampleFormat 1 (unsigned), or 32
// with SampleFormat 3 (IEEE float); Compression 1 (none), 8 or 32946 (Deflate); Predictor 1,
// 2 (horizontal) or 3 (floating point) on Deflate data. Everything else is unsupported_format,
// a strip or tile shorter than its rows is io_error, and `image` is only written on success.
#pragma once

#include <tilestream/sizing.h>
#include <tilestream/types.h>

#include <cstdint>
#include <vector>

namespace tilestream::io {

enum class TiffCompression : std::uint32_t { none, deflate };

// Checked before any pixel memory is allocated: a larger image is resource_limit.
struct TiffReadLimits {
    std::uint32_t max_width = UINT32_MAX;
    std::uint32_t max_height = UINT32_MAX;
    std::uint64_t max_decoded_bytes = max_bytes;
};

// A packed image: rows of width x sample bytes, pitch_bytes apart.
struct TiffImage {
    ImageSpec image;
    std::uint64_t pitch_bytes = 0;
    std::vector<std::uint8_t> pixels;
};

// Tiles are tile_width x tile_height (multiples of 16); edge tiles are padded with zeros.
// horizontal_predictor needs uint16 samples and Deflate; deflate_level is 1-9.
struct TiffWriteOptions {
    bool bigtiff = false;
    TiffCompression compression = TiffCompression::none;
    bool horizontal_predictor = false;
    std::uint32_t tile_width = 128;
    std::uint32_t tile_height = 32;
    std::uint32_t deflate_level = 6;
};

[[nodiscard]] Status read_tiff(const char *path, TiffImage &image,
                               const TiffReadLimits &limits = {}) noexcept;
// A failed write leaves no file behind.
[[nodiscard]] Status write_tiff(const char *path, ConstImageView image,
                                const TiffWriteOptions &options = {}) noexcept;

} // namespace tilestream::io
