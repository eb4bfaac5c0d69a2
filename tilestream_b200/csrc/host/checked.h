// Checked size arithmetic and view validation shared by the host code.
//
// Behaviour follows the reference contracts: every product and sum is checked against
// L = min(INT64_MAX, SIZE_MAX) (src/checked_size.h:9-37, docs/format.md:134), and a view is
// validated in the order image_span -> byte_range -> pointer/alignment -> capacity
// (src/cpu/views.h:9-46), so that each failure maps to the same Status as the reference.
#pragma once

#include <tilestream/format.h>
#include <tilestream/sizing.h>
#include <tilestream/types.h>

#include <cstdint>
#include <cstring>

namespace tilestream::host {

inline bool add(std::uint64_t a, std::uint64_t b, std::uint64_t &out) noexcept {
    if (a > max_bytes || b > max_bytes - a) {
        return false;
    }
    out = a + b;
    return true;
}

inline bool mul(std::uint64_t a, std::uint64_t b, std::uint64_t &out) noexcept {
    if (a > max_bytes || b > max_bytes || (b != 0 && a > max_bytes / b)) {
        return false;
    }
    out = a * b;
    return true;
}

inline bool align_up(std::uint64_t value, std::uint64_t alignment, std::uint64_t &out) noexcept {
    if (alignment == 0 || alignment > max_bytes || value > max_bytes) {
        return false;
    }
    const std::uint64_t rem = value % alignment;
    return add(value, rem == 0 ? 0 : alignment - rem, out);
}

inline bool supported_tile(TileShape t) noexcept {
    return (t.width == 128 && t.height == 32) || (t.width == 64 && t.height == 64) ||
           (t.width == 256 && t.height == 16);
}

// Unsupported type first, then empty dimensions.
inline Status sample_bytes(const ImageSpec &image, std::uint64_t &bytes) noexcept {
    if (image.type != PixelType::uint16 && image.type != PixelType::float32) {
        return Status::unsupported_type;
    }
    if (image.width == 0 || image.height == 0) {
        return Status::invalid_argument;
    }
    bytes = image.type == PixelType::uint16 ? 2 : 4;
    return Status::success;
}

inline std::uint64_t ceil_div(std::uint64_t a, std::uint64_t b) noexcept {
    return a / b + (a % b != 0);
}

inline Status byte_range(const void *data, std::uint64_t capacity) noexcept {
    if (capacity > max_bytes) {
        return Status::size_overflow;
    }
    if (data == nullptr && capacity != 0) {
        return Status::invalid_argument;
    }
    if (capacity > UINTPTR_MAX - reinterpret_cast<std::uintptr_t>(data)) {
        return Status::size_overflow;
    }
    return Status::success;
}

// Both ranges must have passed byte_range.
inline bool overlaps(const void *a, std::uint64_t an, const void *b, std::uint64_t bn) noexcept {
    const auto x = reinterpret_cast<std::uintptr_t>(a);
    const auto y = reinterpret_cast<std::uintptr_t>(b);
    return an != 0 && bn != 0 && x < y + bn && y < x + an;
}

inline Status view_ok(const void *data, const ImageSpec &image, std::uint64_t pitch,
                      std::uint64_t capacity) noexcept {
    std::uint64_t span = 0;
    Status st = image_span(image, pitch, span);
    if (st != Status::success) {
        return st;
    }
    st = byte_range(data, capacity);
    if (st != Status::success) {
        return st;
    }
    const std::uintptr_t alignment = image.type == PixelType::uint16 ? 2 : 4;
    if (data == nullptr || reinterpret_cast<std::uintptr_t>(data) % alignment != 0) {
        return Status::invalid_argument;
    }
    return span <= capacity ? Status::success : Status::buffer_too_small;
}

inline Status view_ok(const ConstImageView &v) noexcept {
    return view_ok(v.data, v.image, v.pitch_bytes, v.capacity_bytes);
}

inline Status view_ok(const ImageView &v) noexcept {
    return view_ok(v.data, v.image, v.pitch_bytes, v.capacity_bytes);
}

// The parser's header rules and statuses (parse_metadata, after reference
// src/cpu/parser.cpp:27-84) for a file of `size` bytes whose first 64 bytes are at `header`
// (size < 64 is malformed_data and reads nothing); on success the image, tile shape and tile
// count. Defined in parser.cpp.
Status check_file_header(const std::uint8_t *header, std::uint64_t size, ImageSpec &image,
                         TileShape &tile, std::uint64_t &tiles) noexcept;

inline std::uint64_t le(const std::uint8_t *p, unsigned n) noexcept {
    std::uint64_t v = 0;
    for (unsigned i = 0; i < n; ++i) {
        v |= std::uint64_t{p[i]} << (8 * i);
    }
    return v;
}

inline void put_le(std::uint8_t *p, std::uint64_t v, unsigned n) noexcept {
    for (unsigned i = 0; i < n; ++i) {
        p[i] = static_cast<std::uint8_t>(v >> (8 * i));
    }
}

inline bool zeros(const std::uint8_t *p, std::uint64_t n) noexcept {
    for (std::uint64_t i = 0; i < n; ++i) {
        if (p[i] != 0) {
            return false;
        }
    }
    return true;
}

// Offsets of the workspace regions of docs/api.md:87-97.
struct WorkspaceLayout {
    std::uint64_t residuals = 0, rows = 0, tiles = 0, lengths = 0, offsets = 0, images = 0,
                  temp = 0, total = 0;
};

[[nodiscard]] Status workspace_layout(const WorkspaceSpec &spec, WorkspaceLayout &out) noexcept;

} // namespace tilestream::host
