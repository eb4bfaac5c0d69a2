// TEST INFRASTRUCTURE ONLY: a C entry layer over the reference's own CPU codec.
//
// oracle/Makefile compiles this file together with the reference sources
// src/sizing.cpp and src/cpu/{parser,encoder,decoder}.cpp, where they lie in the read-only
// reference checkout, into oracle/_ref/libtsref.so. The parity tests use it to pin the C oracle
// to the reference itself, and bench.py times it as the reference CPU baseline. Nothing here is
// part of the product library.
#include <tilestream/api.h>
#include <tilestream/cpu.h>
#include <tilestream/sizing.h>

#include <cstdint>
#include <cstring>

#define TSR_EXPORT extern "C" __attribute__((visibility("default")))

namespace ts = tilestream;

namespace {
ts::ImageSpec spec(std::uint32_t type, std::uint32_t width, std::uint32_t height) {
    return {static_cast<ts::PixelType>(type), width, height};
}
} // namespace

TSR_EXPORT int tsr_compress_bound(std::uint32_t type, std::uint32_t width, std::uint32_t height,
                                  std::uint32_t tw, std::uint32_t th, std::uint64_t *bytes) {
    return static_cast<int>(ts::compress_bound(
        spec(type, width, height),
        {static_cast<std::uint16_t>(tw), static_cast<std::uint16_t>(th)}, *bytes));
}

TSR_EXPORT int tsr_image_span(std::uint32_t type, std::uint32_t width, std::uint32_t height,
                              std::uint64_t pitch, std::uint64_t *bytes) {
    return static_cast<int>(ts::image_span(spec(type, width, height), pitch, *bytes));
}

TSR_EXPORT int tsr_workspace_size(std::uint64_t images, std::uint64_t tiles, std::uint32_t tw,
                                  std::uint32_t th, std::uint64_t temp, std::uint64_t *bytes) {
    ts::WorkspaceSpec s;
    s.image_count = images;
    s.tile_count = tiles;
    s.tile = {static_cast<std::uint16_t>(tw), static_cast<std::uint16_t>(th)};
    s.scan_temp_bytes = temp;
    return static_cast<int>(ts::workspace_size(s, *bytes));
}

TSR_EXPORT int tsr_compress(const void *pixels, std::uint32_t type, std::uint32_t width,
                            std::uint32_t height, std::uint64_t pitch, std::uint64_t capacity,
                            std::uint32_t tw, std::uint32_t th, void *out, std::uint64_t out_size,
                            std::uint64_t *written) {
    return static_cast<int>(ts::cpu::compress(
        {pixels, spec(type, width, height), pitch, capacity},
        {static_cast<std::uint16_t>(tw), static_cast<std::uint16_t>(th)}, {out, out_size},
        *written));
}

// limits: {file_bytes, tile_count, metadata_bytes} or NULL for the defaults.
TSR_EXPORT int tsr_decompress(const void *file, std::uint64_t size, void *pixels,
                              std::uint32_t type, std::uint32_t width, std::uint32_t height,
                              std::uint64_t pitch, std::uint64_t capacity,
                              const std::uint64_t *limits) {
    ts::ParseLimits l;
    if (limits != nullptr) {
        l = {limits[0], limits[1], limits[2]};
    }
    return static_cast<int>(ts::cpu::decompress(
        {file, size}, {pixels, spec(type, width, height), pitch, capacity}, l));
}

// Parses and reports {type, width, height, tile_width, tile_height, file_bytes, tile_count,
// segment_count} in info; tiles/segments (TileMetadata / SegmentMetadata layout) are copied out
// when the pointers are non-null and the capacities suffice.
TSR_EXPORT int tsr_parse(const void *file, std::uint64_t size, const std::uint64_t *limits,
                         std::uint64_t *info, void *tiles, std::uint64_t tile_cap, void *segments,
                         std::uint64_t segment_cap) {
    ts::ParseLimits l;
    if (limits != nullptr) {
        l = {limits[0], limits[1], limits[2]};
    }
    ts::ImageMetadata m;
    const auto status = ts::parse_metadata({file, size}, l, m);
    if (status != ts::Status::success) {
        return static_cast<int>(status);
    }
    info[0] = static_cast<std::uint64_t>(m.image.type);
    info[1] = m.image.width;
    info[2] = m.image.height;
    info[3] = m.tile.width;
    info[4] = m.tile.height;
    info[5] = m.file_bytes;
    info[6] = m.tiles.size();
    info[7] = m.segments.size();
    if (tiles != nullptr && tile_cap >= m.tiles.size() && !m.tiles.empty()) {
        std::memcpy(tiles, m.tiles.data(), m.tiles.size() * sizeof(ts::TileMetadata));
    }
    if (segments != nullptr && segment_cap >= m.segments.size() && !m.segments.empty()) {
        std::memcpy(segments, m.segments.data(), m.segments.size() * sizeof(ts::SegmentMetadata));
    }
    return 0;
}
