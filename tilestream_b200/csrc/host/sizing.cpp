// Size queries of include/tilestream/sizing.h (reference: src/sizing.cpp:9-109). Pure host
// arithmetic; outputs are written only on success.
#include "checked.h"

namespace tilestream {

Status image_span(const ImageSpec &image, std::uint64_t pitch_bytes,
                  std::uint64_t &bytes) noexcept {
    std::uint64_t s = 0;
    const Status st = host::sample_bytes(image, s);
    if (st != Status::success) {
        return st;
    }
    std::uint64_t row = 0;
    if (!host::mul(image.width, s, row) || pitch_bytes > max_bytes) {
        return Status::size_overflow;
    }
    if (pitch_bytes < row || pitch_bytes % s != 0) {
        return Status::invalid_argument;
    }
    std::uint64_t span = 0;
    if (!host::mul(pitch_bytes, std::uint64_t{image.height} - 1, span) ||
        !host::add(span, row, span)) {
        return Status::size_overflow;
    }
    bytes = span;
    return Status::success;
}

// B = 64 + 32 N + W H s + pad, pad = 2 only for uint16 with odd W and odd H
// (docs/format.md:113-132).
Status compress_bound(const ImageSpec &image, TileShape tile, std::uint64_t &bytes) noexcept {
    std::uint64_t s = 0;
    const Status st = host::sample_bytes(image, s);
    if (st != Status::success) {
        return st;
    }
    if (!host::supported_tile(tile)) {
        return Status::invalid_argument;
    }
    const std::uint64_t tiles_x = host::ceil_div(image.width, tile.width);
    const std::uint64_t tiles_y = host::ceil_div(image.height, tile.height);
    const std::uint64_t pad = (s == 2 && image.width % 2 != 0 && image.height % 2 != 0) ? 2 : 0;
    std::uint64_t tiles = 0, index = 0, raw = 0, bound = 0;
    if (!host::mul(tiles_x, tiles_y, tiles) ||
        !host::mul(tiles, format::index_entry_bytes, index) ||
        !host::mul(image.width, image.height, raw) || !host::mul(raw, s, raw) ||
        !host::add(format::header_bytes, index, bound) || !host::add(bound, raw, bound) ||
        !host::add(bound, pad, bound)) {
        return Status::size_overflow;
    }
    bytes = bound;
    return Status::success;
}

Status workspace_size(const WorkspaceSpec &spec, std::uint64_t &bytes) noexcept {
    host::WorkspaceLayout layout;
    const Status st = host::workspace_layout(spec, layout);
    if (st == Status::success) {
        bytes = layout.total;
    }
    return st;
}

namespace host {

// docs/api.md:87-107: seven independent regions, each rounded up to 256 bytes.
Status workspace_layout(const WorkspaceSpec &spec, WorkspaceLayout &out) noexcept {
    if (spec.image_count == 0) {
        if (spec.tile_count != 0 || spec.scan_temp_bytes != 0) {
            return Status::invalid_argument;
        }
        out = {};
        return Status::success;
    }
    if (!supported_tile(spec.tile) || spec.tile_count < spec.image_count) {
        return Status::invalid_argument;
    }
    if (spec.image_count > UINT32_MAX || spec.tile_count > max_window_tiles) {
        return Status::resource_limit;
    }
    WorkspaceLayout r;
    std::uint64_t total = 0;
    auto region = [&total](std::uint64_t count, std::uint64_t size, std::uint64_t &at) {
        std::uint64_t bytes = 0;
        at = total;
        return mul(count, size, bytes) && align_up(bytes, workspace_alignment, bytes) &&
               add(total, bytes, total);
    };
    if (!region(spec.tile_count, 4096 * 4, r.residuals) ||
        !region(spec.tile_count, std::uint64_t{spec.tile.height} * format::segment_header_bytes,
                r.rows) ||
        !region(spec.tile_count, 32, r.tiles) || !region(spec.tile_count, 8, r.lengths) ||
        !region(spec.tile_count + 1, 8, r.offsets) || !region(spec.image_count, 16, r.images) ||
        !region(spec.scan_temp_bytes, 1, r.temp)) {
        return Status::size_overflow;
    }
    r.total = total;
    out = r;
    return Status::success;
}

} // namespace host
} // namespace tilestream
