// Scalar host codec of include/tilestream/cpu.h (reference: src/cpu/encoder.cpp:144-197,
// src/cpu/decoder.cpp:86-110). Produces the canonical bitstream of docs/format.md:99-111 and
// decodes any accepted file. Packing and unpacking work on 64-bit bit buffers instead of single
// bits; the bytes are the same.
#include <tilestream/cpu.h>

#include "checked.h"

#include <algorithm>
#include <cstring>
#include <memory>
#include <new>

namespace tilestream::cpu {
namespace {

using host::le;
using host::put_le;

struct TileWork {
    std::uint32_t samples[4096];
    std::uint32_t residuals[4096];
    std::uint32_t bits[64];
    TileMode mode;
    std::uint64_t length;
};

inline std::uint32_t zigzag16(std::uint32_t cur, std::uint32_t prev) noexcept {
    const std::uint32_t d = (cur - prev) & 0xffffu;
    return d < 32768u ? 2u * d : 2u * (65536u - d) - 1u;
}

template <typename S>
void analyze(const std::uint8_t *origin, std::uint64_t pitch, std::uint32_t w, std::uint32_t h,
             TileWork &t) noexcept {
    constexpr bool f32 = sizeof(S) == 4;
    bool constant = true;
    std::uint64_t predictive = 0;
    std::uint32_t first = 0;
    for (std::uint32_t r = 0; r < h; ++r) {
        const std::uint8_t *line = origin + r * pitch;
        std::uint32_t *px = t.samples + r * w;
        std::uint32_t *res = t.residuals + r * w;
        std::uint32_t any = 0;
        for (std::uint32_t c = 0; c < w; ++c) {
            S v;
            std::memcpy(&v, line + c * sizeof(S), sizeof(S));
            px[c] = v;
        }
        if (r == 0) {
            first = px[0];
        }
        for (std::uint32_t c = 0; c < w; ++c) {
            constant = constant && px[c] == first;
        }
        for (std::uint32_t c = 1; c < w; ++c) {
            const std::uint32_t z = f32 ? (px[c] ^ px[c - 1]) : zigzag16(px[c], px[c - 1]);
            res[c] = z;
            any |= z;
        }
        const std::uint32_t b = any == 0 ? 0u : 32u - static_cast<std::uint32_t>(__builtin_clz(any));
        t.bits[r] = b;
        predictive += 8 + ((std::uint64_t{w} - 1) * b + 31) / 32 * 4;
    }
    t.mode = TileMode::raw;
    t.length = (std::uint64_t{w} * h * sizeof(S) + 3) / 4 * 4;
    if (constant && t.length > 4) {
        t.mode = TileMode::constant;
        t.length = 4;
    }
    if (predictive < t.length) {
        t.mode = TileMode::predict_bitpack;
        t.length = predictive;
    }
}

template <typename S>
void write_tile(std::uint8_t *out, const TileWork &t, std::uint32_t w, std::uint32_t h) noexcept {
    std::memset(out, 0, static_cast<std::size_t>(t.length));
    if (t.mode == TileMode::raw) {
        for (std::uint32_t i = 0; i < w * h; ++i) {
            put_le(out + i * sizeof(S), t.samples[i], sizeof(S));
        }
        return;
    }
    if (t.mode == TileMode::constant) {
        put_le(out, t.samples[0], sizeof(S));
        return;
    }
    for (std::uint32_t r = 0; r < h; ++r) {
        const std::uint32_t b = t.bits[r];
        put_le(out, t.samples[r * w], 4);
        out[4] = static_cast<std::uint8_t>(b);
        out += format::segment_header_bytes;
        const std::uint32_t *res = t.residuals + r * w;
        std::uint64_t buffer = 0;
        unsigned filled = 0;
        std::uint8_t *word = out;
        for (std::uint32_t c = 1; c < w; ++c) {
            buffer |= std::uint64_t{res[c]} << filled;
            filled += b;
            if (filled >= 32) {
                put_le(word, static_cast<std::uint32_t>(buffer), 4);
                word += 4;
                buffer >>= 32;
                filled -= 32;
            }
        }
        if (filled != 0) {
            put_le(word, static_cast<std::uint32_t>(buffer), 4);
        }
        out += (std::uint64_t{w - 1} * b + 31) / 32 * 4;
    }
}

void write_header(std::uint8_t *o, const ImageSpec &image, TileShape tile, std::uint64_t count,
                  std::uint64_t size) noexcept {
    std::memset(o, 0, format::header_bytes);
    std::copy(format::magic.begin(), format::magic.end(), o);
    put_le(o + format::header::version_major, format::major_version, 2);
    put_le(o + format::header::version_minor, format::minor_version, 2);
    put_le(o + format::header::size, format::header_bytes, 2);
    o[format::header::pixel_type] = static_cast<std::uint8_t>(image.type);
    put_le(o + format::header::width, image.width, 4);
    put_le(o + format::header::height, image.height, 4);
    put_le(o + format::header::tile_width, tile.width, 2);
    put_le(o + format::header::tile_height, tile.height, 2);
    put_le(o + format::header::entry_size, format::index_entry_bytes, 2);
    put_le(o + format::header::tile_count, count, 8);
    put_le(o + format::header::index_offset, format::header_bytes, 8);
    put_le(o + format::header::payload_offset,
           format::header_bytes + count * format::index_entry_bytes, 8);
    put_le(o + format::header::file_size, size, 8);
}

template <typename S>
std::uint64_t encode(const ConstImageView &in, TileShape tile, std::uint8_t *out,
                     TileWork &work) noexcept {
    const ImageSpec &im = in.image;
    const std::uint64_t across = host::ceil_div(im.width, tile.width);
    const std::uint64_t count = across * host::ceil_div(im.height, tile.height);
    std::uint64_t cursor = format::header_bytes + count * format::index_entry_bytes;
    const auto *base = static_cast<const std::uint8_t *>(in.data);
    for (std::uint64_t i = 0; i < count; ++i) {
        const std::uint64_t x = (i % across) * tile.width;
        const std::uint64_t y = (i / across) * tile.height;
        const auto w = static_cast<std::uint32_t>(std::min<std::uint64_t>(tile.width, im.width - x));
        const auto h =
            static_cast<std::uint32_t>(std::min<std::uint64_t>(tile.height, im.height - y));
        analyze<S>(base + y * in.pitch_bytes + x * sizeof(S), in.pitch_bytes, w, h, work);
        std::uint8_t *e = out + format::header_bytes + i * format::index_entry_bytes;
        std::memset(e, 0, format::index_entry_bytes);
        e[format::entry::mode] = static_cast<std::uint8_t>(work.mode);
        put_le(e + format::entry::width, w, 2);
        put_le(e + format::entry::height, h, 2);
        put_le(e + format::entry::offset, cursor, 8);
        put_le(e + format::entry::length, work.length, 8);
        write_tile<S>(out + cursor, work, w, h);
        cursor += work.length;
    }
    write_header(out, im, tile, count, cursor);
    return cursor;
}

// One b-bit residual j of a row (docs/format.md:77-79): a second word is read only when the
// symbol crosses into it, and neither b = 0 nor b = 32 shifts by 32.
inline std::uint32_t symbol(const std::uint8_t *packed, std::uint64_t j, std::uint32_t b) noexcept {
    if (b == 0) {
        return 0;
    }
    if (b == 32) {
        return static_cast<std::uint32_t>(le(packed + 4 * j, 4));
    }
    const std::uint64_t pos = j * b;
    const std::uint32_t shift = static_cast<std::uint32_t>(pos % 32);
    const std::uint8_t *word = packed + pos / 32 * 4;
    std::uint32_t v = static_cast<std::uint32_t>(le(word, 4)) >> shift;
    if (shift + b > 32) {
        v |= static_cast<std::uint32_t>(le(word + 4, 4)) << (32 - shift);
    }
    return v & ((1u << b) - 1u);
}

template <typename S>
void decode(const std::uint8_t *file, const ImageMetadata &m, const ImageView &out) noexcept {
    constexpr bool f32 = sizeof(S) == 4;
    const std::uint64_t across = host::ceil_div(m.image.width, m.tile.width);
    auto *base = static_cast<std::uint8_t *>(out.data);
    for (std::size_t i = 0; i < m.tiles.size(); ++i) {
        const TileMetadata &t = m.tiles[i];
        const std::uint64_t x = (i % across) * m.tile.width;
        const std::uint64_t y = (i / across) * m.tile.height;
        const std::uint8_t *p = file + t.offset;
        for (std::uint32_t r = 0; r < t.height; ++r) {
            std::uint8_t *line = base + (y + r) * out.pitch_bytes + x * sizeof(S);
            if (t.mode == TileMode::raw) {
                std::memcpy(line, p + std::uint64_t{r} * t.width * sizeof(S), t.width * sizeof(S));
            } else if (t.mode == TileMode::constant) {
                const S v = static_cast<S>(le(p, sizeof(S)));
                for (std::uint32_t c = 0; c < t.width; ++c) {
                    std::memcpy(line + c * sizeof(S), &v, sizeof(S));
                }
            } else {
                const SegmentMetadata &g = m.segments[t.first_segment + r];
                const std::uint8_t *packed = p + g.payload_offset;
                std::uint32_t value = g.seed;
                S v = static_cast<S>(value);
                std::memcpy(line, &v, sizeof(S));
                for (std::uint32_t c = 1; c < t.width; ++c) {
                    const std::uint32_t z = symbol(packed, c - 1, g.bit_width);
                    value = f32 ? value ^ z : (value + ((z >> 1) ^ (0u - (z & 1u)))) & 0xffffu;
                    v = static_cast<S>(value);
                    std::memcpy(line + c * sizeof(S), &v, sizeof(S));
                }
            }
        }
    }
}

} // namespace

Status compress(ConstImageView input, TileShape tile, MutableBytes output,
                std::uint64_t &bytes_written) noexcept {
    Status st = host::view_ok(input);
    if (st != Status::success) {
        return st;
    }
    std::uint64_t bound = 0;
    st = compress_bound(input.image, tile, bound);
    if (st != Status::success) {
        return st;
    }
    st = host::byte_range(output.data, output.size);
    if (st != Status::success) {
        return st;
    }
    if (output.size < bound) {
        return Status::buffer_too_small;
    }
    if (host::overlaps(input.data, input.capacity_bytes, output.data, output.size) ||
        host::overlaps(&bytes_written, sizeof(bytes_written), output.data, output.size) ||
        host::overlaps(&bytes_written, sizeof(bytes_written), input.data, input.capacity_bytes)) {
        return Status::invalid_argument;
    }
    std::unique_ptr<TileWork> work(new (std::nothrow) TileWork);
    if (!work) {
        return Status::resource_limit;
    }
    auto *out = static_cast<std::uint8_t *>(output.data);
    bytes_written = input.image.type == PixelType::uint16
                        ? encode<std::uint16_t>(input, tile, out, *work)
                        : encode<std::uint32_t>(input, tile, out, *work);
    return Status::success;
}

Status decompress(ConstBytes input, ImageView output, const ParseLimits &limits) noexcept {
    Status st = host::view_ok(output);
    if (st != Status::success) {
        return st;
    }
    st = host::byte_range(input.data, input.size);
    if (st != Status::success) {
        return st;
    }
    if (host::overlaps(input.data, input.size, output.data, output.capacity_bytes)) {
        return Status::invalid_argument;
    }
    ImageMetadata m;
    st = parse_metadata(input, limits, m);
    if (st != Status::success) {
        return st;
    }
    if (output.image.width != m.image.width || output.image.height != m.image.height ||
        output.image.type != m.image.type) {
        return Status::invalid_argument;
    }
    const auto *file = static_cast<const std::uint8_t *>(input.data);
    if (m.image.type == PixelType::uint16) {
        decode<std::uint16_t>(file, m, output);
    } else {
        decode<std::uint32_t>(file, m, output);
    }
    return Status::success;
}

} // namespace tilestream::cpu
