#pragma once
// Drop-in replacement for the reference's include/tilestream/api.h (api.h:1-45):
// host metadata produced by the untrusted-file parser.
#include <tilestream/sizing.h>
#include <tilestream/types.h>

#include <cstdint>
#include <vector>

namespace tilestream {

struct SegmentMetadata {
    std::uint32_t seed = 0;
    std::uint32_t bit_width = 0;
    std::uint64_t payload_offset = 0; // Packed words, relative to the tile's payload start.
    std::uint64_t payload_bytes = 0;
};

struct TileMetadata {
    TileMode mode = TileMode::raw;
    std::uint16_t width = 0;
    std::uint16_t height = 0;
    std::uint64_t offset = 0; // Absolute byte offset in the file.
    std::uint64_t length = 0;
    std::uint64_t first_segment = 0;
};

struct ImageMetadata {
    ImageSpec image;
    TileShape tile;
    std::uint64_t file_bytes = 0;
    std::vector<TileMetadata> tiles;
    std::vector<SegmentMetadata> segments;
};

// Caller budgets checked before the parser allocates its tables.
struct ParseLimits {
    std::uint64_t file_bytes = max_bytes;
    std::uint64_t tile_count = max_bytes;
    std::uint64_t metadata_bytes = max_bytes;
};

// Validates a complete uint16 or bit-exact FP32 archive; metadata is untouched on failure.
[[nodiscard]] Status parse_metadata(ConstBytes source, const ParseLimits &limits,
                                    ImageMetadata &metadata) noexcept;

} // namespace tilestream
