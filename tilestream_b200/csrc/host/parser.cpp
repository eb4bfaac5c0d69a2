// Untrusted .tsc parser (include/tilestream/api.h; reference: src/cpu/parser.cpp:27-242).
//
// Validation order and status mapping follow docs/format.md:136-147 and docs/api.md:43-47:
// the fixed header first, then the caller's budgets, then every index entry, payload and row
// descriptor (lengths before contents, widths before arithmetic), then the native tables are
// filled. The budget counts native table bytes; sizeof values below are those of the public
// records. On failure the caller's metadata is untouched.
//
// The reference walks every payload twice (once to count row segments, once to fill the
// tables). Here the index is checked first, which fixes the segment count (one per row of
// every PREDICT tile) and where each tile's segments go, and the payloads are walked once, with
// word loads, split over up to 8 host threads (TILESTREAM_PARSE_THREADS) for files of at least
// 1024 tiles.
#include <tilestream/api.h>

#include "checked.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>
#include <new>
#include <stdexcept>
#include <utility>

namespace tilestream {
namespace {

using host::le;
using host::zeros;

struct Header {
    ImageSpec image;
    TileShape tile;
    std::uint64_t across = 0;
    std::uint64_t count = 0;
    std::uint64_t payload = 0;
};

Status read_header(const std::uint8_t *d, std::uint64_t size, Header &h) noexcept {
    if (size < format::header_bytes) {
        return Status::malformed_data;
    }
    for (std::size_t i = 0; i < format::magic.size(); ++i) {
        if (d[i] != format::magic[i]) {
            return Status::malformed_data;
        }
    }
    if (le(d + format::header::version_major, 2) != format::major_version ||
        le(d + format::header::version_minor, 2) != format::minor_version ||
        d[format::header::flags] != 0) {
        return Status::unsupported_format;
    }
    if (le(d + format::header::size, 2) != format::header_bytes ||
        le(d + format::header::entry_size, 2) != format::index_entry_bytes ||
        !zeros(d + format::header::reserved, 2)) {
        return Status::malformed_data;
    }
    const std::uint8_t type = d[format::header::pixel_type];
    if (type != static_cast<std::uint8_t>(PixelType::uint16) &&
        type != static_cast<std::uint8_t>(PixelType::float32)) {
        return Status::unsupported_type;
    }
    h.image = {static_cast<PixelType>(type),
               static_cast<std::uint32_t>(le(d + format::header::width, 4)),
               static_cast<std::uint32_t>(le(d + format::header::height, 4))};
    h.tile = {static_cast<std::uint16_t>(le(d + format::header::tile_width, 2)),
              static_cast<std::uint16_t>(le(d + format::header::tile_height, 2))};
    if (h.image.width == 0 || h.image.height == 0) {
        return Status::malformed_data;
    }
    if (!host::supported_tile(h.tile)) {
        return Status::unsupported_format;
    }
    std::uint64_t bound = 0;
    const Status st = compress_bound(h.image, h.tile, bound);
    if (st != Status::success) {
        return st;
    }
    h.across = host::ceil_div(h.image.width, h.tile.width);
    const std::uint64_t down = host::ceil_div(h.image.height, h.tile.height);
    std::uint64_t index = 0;
    if (!host::mul(h.across, down, h.count) ||
        !host::mul(h.count, format::index_entry_bytes, index) ||
        !host::add(format::header_bytes, index, h.payload)) {
        return Status::size_overflow;
    }
    if (le(d + format::header::tile_count, 8) != h.count ||
        le(d + format::header::index_offset, 8) != format::header_bytes ||
        le(d + format::header::payload_offset, 8) != h.payload ||
        le(d + format::header::file_size, 8) != size || size > bound || h.payload > size) {
        return Status::malformed_data;
    }
    return Status::success;
}

// Little-endian loads of the payload words (the host is little-endian, as the format).
static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__, "little-endian host");
inline std::uint32_t load32(const std::uint8_t *p) noexcept {
    std::uint32_t v;
    std::memcpy(&v, p, 4);
    return v;
}

// Tile i's geometry: its width and height.
struct TileSize {
    std::uint64_t w, h;
};
inline TileSize tile_size(const Header &h, std::uint64_t i) noexcept {
    const std::uint64_t x = (i % h.across) * h.tile.width;
    const std::uint64_t y = (i / h.across) * h.tile.height;
    return {std::min<std::uint64_t>(h.tile.width, h.image.width - x),
            std::min<std::uint64_t>(h.tile.height, h.image.height - y)};
}

// Validates every index entry: mode, reserved bytes, geometry, and lengths against the
// payload chain and the tile's RAW size. A PREDICT tile has one row segment per row, so the
// number of segments is known from the index alone.
Status check_index(const std::uint8_t *d, std::uint64_t size, const Header &h,
                   std::uint64_t &segments) noexcept {
    const std::uint64_t s = h.image.type == PixelType::uint16 ? 2 : 4;
    std::uint64_t expected = h.payload;
    std::uint64_t nseg = 0;
    for (std::uint64_t i = 0; i < h.count; ++i) {
        const std::uint8_t *e = d + format::header_bytes + i * format::index_entry_bytes;
        const TileSize t = tile_size(h, i);
        const std::uint64_t offset = le(e + format::entry::offset, 8);
        const std::uint64_t length = le(e + format::entry::length, 8);
        const std::uint64_t raw4 = (t.w * t.h * s + 3) / 4 * 4;
        const std::uint8_t mode = e[format::entry::mode];
        if (mode > static_cast<std::uint8_t>(TileMode::predict_bitpack) ||
            !zeros(e + format::entry::reserved, 3) || !zeros(e + format::entry::reserved_tail, 8) ||
            le(e + format::entry::width, 2) != t.w || le(e + format::entry::height, 2) != t.h ||
            offset != expected || offset > size || length > size - offset || length == 0 ||
            length % 4 != 0 || length > raw4) {
            return Status::malformed_data;
        }
        if (mode == 2) {
            nseg += t.h;
        }
        expected += length;
    }
    segments = nseg;
    return expected == size ? Status::success : Status::malformed_data;
}

// Validates the payloads of tiles [begin, end) of a file whose index check_index accepted;
// `nseg` is the number of row segments of the tiles before `begin`. With out != nullptr (tables
// sized by check_index) it also fills their tile and segment records.
Status check_payloads(const std::uint8_t *d, const Header &h, ImageMetadata *out,
                      std::uint64_t begin, std::uint64_t end, std::uint64_t nseg) noexcept {
    const std::uint64_t s = h.image.type == PixelType::uint16 ? 2 : 4;
    const std::uint32_t max_bits = h.image.type == PixelType::uint16 ? 16 : 32;
    for (std::uint64_t i = begin; i < end; ++i) {
        const std::uint8_t *e = d + format::header_bytes + i * format::index_entry_bytes;
        const TileSize t = tile_size(h, i);
        const std::uint64_t offset = le(e + format::entry::offset, 8);
        const std::uint64_t length = le(e + format::entry::length, 8);
        const std::uint64_t raw = t.w * t.h * s;
        const std::uint64_t raw4 = (raw + 3) / 4 * 4;
        const std::uint8_t mode = e[format::entry::mode];
        const std::uint8_t *p = d + offset;
        const std::uint64_t first = mode == 2 ? nseg : 0;
        if (mode == 0) {
            if (length != raw4 || !zeros(p + raw, length - raw)) {
                return Status::malformed_data;
            }
        } else if (mode == 1) {
            if (length != 4 || (s == 2 && !zeros(p + 2, 2))) {
                return Status::malformed_data;
            }
        } else {
            std::uint64_t cursor = 0;
            for (std::uint64_t r = 0; r < t.h; ++r) {
                if (length - cursor < format::segment_header_bytes) {
                    return Status::malformed_data;
                }
                const std::uint8_t *desc = p + cursor;
                const std::uint32_t seed = load32(desc + format::segment::seed);
                // Width byte, then three reserved zero bytes: one little-endian word.
                const std::uint32_t word = load32(desc + format::segment::bit_width);
                const std::uint32_t bits = word & 0xffu;
                if ((s == 2 && seed > UINT16_MAX) || bits > max_bits || (t.w == 1 && bits != 0) ||
                    (word >> 8) != 0) {
                    return Status::malformed_data;
                }
                cursor += format::segment_header_bytes;
                const std::uint64_t nbits = (t.w - 1) * bits;
                const std::uint64_t packed = (nbits + 31) / 32 * 4;
                if (packed > length - cursor) {
                    return Status::malformed_data;
                }
                // Unused high bits of the last word must be zero.
                if (nbits % 32 != 0 && (load32(p + cursor + packed - 4) >> (nbits % 32)) != 0) {
                    return Status::malformed_data;
                }
                if (out != nullptr) {
                    out->segments[nseg] = {seed, bits, cursor, packed};
                }
                ++nseg;
                cursor += packed;
            }
            if (cursor != length) {
                return Status::malformed_data;
            }
        }
        if (out != nullptr) {
            out->tiles[i] = {static_cast<TileMode>(mode), static_cast<std::uint16_t>(t.w),
                             static_cast<std::uint16_t>(t.h), offset, length, first};
        }
    }
    return Status::success;
}

// Row segments of the tiles before tile `end` (from the index, which check_index accepted).
std::uint64_t segments_before(const std::uint8_t *d, const Header &h, std::uint64_t end) noexcept {
    std::uint64_t nseg = 0;
    for (std::uint64_t i = 0; i < end; ++i) {
        if (d[format::header_bytes + i * format::index_entry_bytes + format::entry::mode] == 2) {
            nseg += tile_size(h, i).h;
        }
    }
    return nseg;
}

// Threads a parse may use: TILESTREAM_PARSE_THREADS when set (1 keeps every parse on the
// calling thread, for processes that parse on many threads already), else up to 8 of the
// host's cores. Read once per process.
std::uint64_t parse_threads() noexcept {
    static const std::uint64_t threads = [] {
        const char *v = std::getenv("TILESTREAM_PARSE_THREADS");
        if (v != nullptr && *v != 0) {
            const long n = std::strtol(v, nullptr, 10);
            return static_cast<std::uint64_t>(n < 1 ? 1 : (n > 64 ? 64 : n));
        }
        const unsigned cores = std::thread::hardware_concurrency();
        return static_cast<std::uint64_t>(cores == 0 ? 1 : std::min(cores, 8u));
    }();
    return threads;
}

// All payloads. A large file is cut into ranges of whole tiles checked on a few host threads
// (each range knows its first segment from the index); with fewer tiles, or when a thread
// cannot be started, the ranges run on the calling thread. Every failure is malformed_data,
// so it does not matter which range finds one first.
Status check_all_payloads(const std::uint8_t *d, const Header &h, ImageMetadata *out) noexcept {
    constexpr std::uint64_t kMinTilesPerThread = 512;
    std::uint64_t parts = parse_threads();
    parts = std::max<std::uint64_t>(1, std::min<std::uint64_t>(parts, h.count / kMinTilesPerThread));
    if (parts == 1) {
        return check_payloads(d, h, out, 0, h.count, 0);
    }
    std::vector<Status> status;
    std::vector<std::thread> pool;
    try {
        status.assign(parts, Status::success);
    } catch (...) {
        return check_payloads(d, h, out, 0, h.count, 0);
    }
    std::uint64_t started = 0;
    auto range = [&](std::uint64_t k) {
        const std::uint64_t begin = h.count * k / parts, end = h.count * (k + 1) / parts;
        status[k] = check_payloads(d, h, out, begin, end, segments_before(d, h, begin));
    };
    try {
        pool.reserve(parts - 1);
        for (std::uint64_t k = 1; k < parts; ++k) {
            pool.emplace_back(range, k);
            started = k;
        }
    } catch (...) {
        // Fewer threads than planned: the calling thread takes the rest below.
    }
    range(0);
    for (std::uint64_t k = started + 1; k < parts; ++k) {
        range(k);
    }
    for (auto &t : pool) {
        t.join();
    }
    for (const Status st : status) {
        if (st != Status::success) {
            return st;
        }
    }
    return Status::success;
}

Status table_bytes(std::uint64_t tiles, std::uint64_t segments, std::uint64_t &bytes) noexcept {
    std::uint64_t t = 0, g = 0, total = 0;
    if (!host::mul(tiles, sizeof(TileMetadata), t) ||
        !host::mul(segments, sizeof(SegmentMetadata), g) ||
        !host::add(sizeof(ImageMetadata), t, total) || !host::add(total, g, total)) {
        return Status::size_overflow;
    }
    bytes = total;
    return Status::success;
}

} // namespace

namespace host {

Status check_file_header(const std::uint8_t *header, std::uint64_t size, ImageSpec &image,
                         TileShape &tile, std::uint64_t &tiles) noexcept {
    Header h;
    const Status st = read_header(header, size, h);
    if (st == Status::success) {
        image = h.image;
        tile = h.tile;
        tiles = h.count;
    }
    return st;
}

} // namespace host

Status parse_metadata(ConstBytes source, const ParseLimits &limits,
                      ImageMetadata &metadata) noexcept {
    Status st = host::byte_range(source.data, source.size);
    if (st != Status::success) {
        return st;
    }
    if (source.size > limits.file_bytes) {
        return Status::resource_limit;
    }
    const auto *d = static_cast<const std::uint8_t *>(source.data);
    Header h;
    st = read_header(d, source.size, h);
    if (st != Status::success) {
        return st;
    }
    if (h.count > limits.tile_count) {
        return Status::resource_limit;
    }
    std::uint64_t need = 0;
    st = table_bytes(h.count, 0, need);
    if (st != Status::success) {
        return st;
    }
    if (need > limits.metadata_bytes) {
        return Status::resource_limit;
    }
    // The index first (it also gives the exact number of row segments), then the budget, then
    // one pass over the payloads that validates them and fills the tables. Every failure of
    // the two checks is malformed_data, so checking all entries before any payload reports
    // what a tile-by-tile walk would; a file over budget still has its payloads checked first,
    // so malformed_data keeps precedence over resource_limit.
    std::uint64_t segments = 0;
    st = check_index(d, source.size, h, segments);
    if (st != Status::success) {
        return st;
    }
    st = table_bytes(h.count, segments, need);
    if (st != Status::success || need > limits.metadata_bytes) {
        const Status payloads = check_all_payloads(d, h, nullptr);
        if (payloads != Status::success) {
            return payloads;
        }
        return st != Status::success ? st : Status::resource_limit;
    }
    try {
        ImageMetadata parsed;
        parsed.image = h.image;
        parsed.tile = h.tile;
        parsed.file_bytes = source.size;
        parsed.tiles.resize(static_cast<std::size_t>(h.count));
        parsed.segments.resize(static_cast<std::size_t>(segments));
        st = check_all_payloads(d, h, &parsed);
        if (st != Status::success) {
            return st;
        }
        metadata = std::move(parsed);
        return Status::success;
    } catch (const std::bad_alloc &) {
        return Status::resource_limit;
    } catch (const std::length_error &) {
        return Status::resource_limit;
    }
}

} // namespace tilestream
