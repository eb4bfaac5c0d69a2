// TEST INFRASTRUCTURE ONLY: deterministic test inputs for the oracle-based parity tests.
//
// Restates the reference's seeded robustness generator (tests/robustness/cases.h:38-170) and the
// corpus-driven file mutator of its fuzz harness (fuzz/harness.h:190-307), so that the parity
// tests draw exactly the reference's cases from the same seeds and rebuild the reference's
// mutation corpus inputs as .tsc files. Both use std::mt19937_64, which the C++ standard defines
// bit-exactly. Encoding and parsing inside the mutator go through the C oracle.
#include "tsc_oracle.h"

#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

namespace {

constexpr std::uint64_t kFirstSeed = 13000000; // cases.h:21
constexpr std::uint32_t kShapes[3][2] = {{128, 32}, {64, 64}, {256, 16}};
constexpr std::uint32_t kSpecial[] = {0x00000000, 0x80000000, 0x00000001, 0x807fffff,
                                      0x00800000, 0x7f7fffff, 0xff800000, 0x7f800000,
                                      0x7fc00000, 0xffc12345, 0x7f800001, 0x3f800000};

// cases.h:38-94. Eight patterns; the number of engine draws per pixel depends on the pattern,
// exactly as in the reference.
void fill(std::uint32_t type, std::uint32_t width, std::uint32_t height, std::uint64_t pitch,
          std::uint32_t pattern, std::uint64_t seed, std::uint8_t *bytes) {
    std::mt19937_64 rng(seed);
    const std::uint64_t s = type == TSO_UINT16 ? 2 : 4;
    const std::uint32_t mask = type == TSO_UINT16 ? 0xffffU : 0xffffffffU;
    const auto base = static_cast<std::uint32_t>(rng());
    const auto bits = static_cast<std::uint32_t>(rng() % (type == TSO_UINT16 ? 17 : 33));
    const std::uint32_t spread = bits == 32 ? 0xffffffffU : (1U << bits) - 1;
    for (std::uint32_t y = 0; y < height; ++y) {
        std::uint32_t previous = base;
        for (std::uint32_t x = 0; x < width; ++x) {
            std::uint32_t value = 0;
            switch (pattern % 8) {
            case 0:
                value = base;
                break;
            case 1:
                value = base + x * 3 + y * 7;
                break;
            case 2:
                value = 65535U - x - y * width;
                break;
            case 3: {
                const auto r = static_cast<std::uint32_t>(rng()) & spread;
                value = type == TSO_UINT16 ? previous + r : previous ^ r;
                break;
            }
            case 4:
                value = static_cast<std::uint32_t>(rng());
                break;
            case 5: {
                // The FP32 field draws once; the uint16 branch draws a second time.
                const float field = 1.5F + 0.001F * static_cast<float>(x) +
                                    0.01F * static_cast<float>(y) +
                                    0.0001F * static_cast<float>(rng() % 7);
                if (type == TSO_UINT16) {
                    value = 1000 + x / 4 + y / 8 + static_cast<std::uint32_t>(rng() % 16);
                } else {
                    std::memcpy(&value, &field, 4);
                }
                break;
            }
            case 6:
                value = type == TSO_UINT16 ? (rng() % 2 == 0 ? 0U : 65535U)
                                           : kSpecial[rng() % (sizeof(kSpecial) / 4)];
                break;
            default:
                value = (x / 8 + y / 4) % 2 == 0 ? base : base ^ (1U << (rng() % 32));
                break;
            }
            previous = value & mask;
            std::memcpy(bytes + y * pitch + x * s, &previous, static_cast<std::size_t>(s));
        }
    }
}

// cases.h:134-144.
std::uint32_t pick_size(std::mt19937_64 &rng, std::uint32_t limit) {
    static constexpr std::uint32_t edges[] = {1,  2,   3,   31,  32,  33,  63, 64,
                                              65, 127, 128, 129, 255, 256, 257};
    if (rng() % 2 == 0) {
        const auto value = edges[rng() % 15];
        if (value <= limit) {
            return value;
        }
    }
    return 1 + static_cast<std::uint32_t>(rng() % limit);
}

struct Reader {
    const std::uint8_t *data;
    std::size_t size;
    std::size_t position = 0;
    bool empty() const { return position >= size; }
    std::uint64_t take(std::uint64_t bytes) {
        std::uint64_t value = 0;
        for (std::uint64_t i = 0; i < bytes && position < size; ++i) {
            value |= std::uint64_t{data[position++]} << (8 * i);
        }
        return value;
    }
};

std::uint64_t rd(const std::uint8_t *p, std::uint64_t n) {
    std::uint64_t v = 0;
    for (std::uint64_t i = 0; i < n; ++i) v |= std::uint64_t{p[i]} << (8 * i);
    return v;
}

void wr(std::uint8_t *p, std::uint64_t n, std::uint64_t v) {
    for (std::uint64_t i = 0; i < n; ++i) p[i] = static_cast<std::uint8_t>(v >> (8 * i));
}

struct Field {
    std::uint64_t offset, bytes;
};
constexpr Field kHeader[] = {{0, 8},  {8, 2},  {10, 2}, {12, 2}, {14, 1}, {15, 1},
                             {16, 4}, {20, 4}, {24, 2}, {26, 2}, {28, 2}, {30, 2},
                             {32, 8}, {40, 8}, {48, 8}, {56, 8}};
constexpr Field kEntry[] = {{0, 1}, {1, 3}, {4, 2}, {6, 2}, {8, 8}, {16, 8}, {24, 8}};
constexpr Field kSegment[] = {{0, 4}, {4, 1}, {5, 3}};

// harness.h:169-175: replace a field, or move it by a signed byte when bit 63 is set.
void change(std::vector<std::uint8_t> &file, std::uint64_t at, Field f, std::uint64_t value) {
    if (at + f.bytes > file.size()) return;
    const auto old = rd(file.data() + at, f.bytes);
    const auto delta = static_cast<std::uint64_t>(static_cast<std::int8_t>(value & 0xff));
    wr(file.data() + at, f.bytes, (value >> 63) != 0 ? old + delta : value >> 8);
}

// harness.h:177-207: grow or shrink one tile payload by whole words, shifting later offsets.
void splice(std::vector<std::uint8_t> &file, std::uint64_t tiles, std::uint64_t index,
            std::uint64_t field, std::uint64_t value) {
    if (file.size() < 64 + 32 * tiles) return;
    const auto entry = 64 + 32 * index;
    const auto offset = rd(file.data() + entry + 8, 8);
    const auto length = rd(file.data() + entry + 16, 8);
    const auto bytes = 4 * (1 + field % 4);
    const bool grow = value % 2 == 0;
    if (offset > file.size() || length > file.size() - offset || (!grow && length < bytes)) return;
    const auto end = file.begin() + static_cast<std::ptrdiff_t>(offset + length);
    if (grow) {
        file.insert(end, bytes, static_cast<std::uint8_t>(value >> 8));
    } else {
        file.erase(end - static_cast<std::ptrdiff_t>(bytes), end);
    }
    const auto delta = grow ? bytes : 0 - bytes;
    wr(file.data() + entry + 16, 8, length + delta);
    for (auto i = index + 1; i < tiles; ++i) {
        auto *later = file.data() + 64 + 32 * i + 8;
        wr(later, 8, rd(later, 8) + delta);
    }
    wr(file.data() + 56, 8, rd(file.data() + 56, 8) + delta);
}

} // namespace

extern "C" {

// cases.h:147-170. info receives {type, width, height, tile_width, tile_height, pattern,
// roi_x, roi_y, roi_width, roi_height}. With bytes == NULL only the description is produced;
// otherwise bytes receives pitch * height bytes (0x5a padding, then the pixels).
void tso_case(std::uint64_t seed, std::uint32_t *info, std::uint64_t *pitch,
              std::uint8_t *bytes) {
    const auto index = seed - kFirstSeed;
    std::mt19937_64 rng(seed);
    const std::uint32_t type = index % 2 == 0 ? TSO_UINT16 : TSO_FLOAT32;
    const auto *shape = kShapes[index / 2 % 3];
    const std::uint32_t width = pick_size(rng, 300);
    const std::uint32_t height = pick_size(rng, 160);
    const std::uint64_t s = type == TSO_UINT16 ? 2 : 4;
    const std::uint64_t padding = rng() % 4 == 0 ? rng() % 5 : 0;
    const std::uint64_t p = (width + padding) * s;
    const auto pattern = static_cast<std::uint32_t>(rng() % 8);
    std::uint32_t roi[4] = {0, 0, width, height};
    if (rng() % 4 != 0) {
        roi[0] = static_cast<std::uint32_t>(rng() % width);
        roi[1] = static_cast<std::uint32_t>(rng() % height);
        roi[2] = 1 + static_cast<std::uint32_t>(rng() % (width - roi[0]));
        roi[3] = 1 + static_cast<std::uint32_t>(rng() % (height - roi[1]));
    }
    const std::uint64_t fill_seed = rng();
    const std::uint32_t values[10] = {type,   width,  height, shape[0], shape[1],
                                      pattern, roi[0], roi[1], roi[2],   roi[3]};
    std::memcpy(info, values, sizeof(values));
    *pitch = p;
    if (bytes != nullptr) {
        std::memset(bytes, 0x5a, static_cast<std::size_t>(p * height));
        fill(type, width, height, p, pattern, fill_seed, bytes);
    }
}

// The robustness fill pattern alone (cases.h:38-94), for tests that pick their own shapes.
void tso_fill(std::uint32_t type, std::uint32_t width, std::uint32_t height, std::uint64_t pitch,
              std::uint32_t pattern, std::uint64_t seed, std::uint8_t *bytes) {
    fill(type, width, height, pitch, pattern, seed, bytes);
}

// ---- fabricated metadata (tests/cuda_robustness_test.cpp:194-243) -------------------------
// One std::mt19937_64 engine that the Python side draws from between fabrications (the ROI of
// each trial), so the whole campaign consumes the engine in the reference test's order.
void *tso_rng_new(std::uint64_t seed) {
    return new std::mt19937_64(seed);
}
void tso_rng_free(void *rng) {
    delete static_cast<std::mt19937_64 *>(rng);
}
std::uint64_t tso_rng_next(void *rng) {
    return (*static_cast<std::mt19937_64 *>(rng))();
}

// Host metadata records with the layout of the library's TileMetadata (32 bytes) and
// SegmentMetadata (24 bytes).
struct FabTile {
    std::uint32_t mode;
    std::uint16_t width, height;
    std::uint64_t offset, length, first_segment;
};
struct FabSegment {
    std::uint32_t seed, bit_width;
    std::uint64_t payload_offset, payload_bytes;
};

// A field moved by a small multiple of `step`, or (one time in three) replaced by an arbitrary
// value: 64 random bits one time in three of those, else a value below 65536. Arithmetic is
// modulo 2^64, as in the reference.
static std::uint64_t nudge(std::uint64_t value, std::mt19937_64 &rng, std::uint64_t step) {
    if (rng() % 3 == 0) {
        if (rng() % 3 == 0) return rng();
        return rng() % 65536;
    }
    const std::uint64_t k = rng() % 17;
    return value + (k - 8) * step;
}

// Changes one field of the metadata, drawing in the reference's order: the tile, then the
// segment (a default segment is appended when there is none), then the field among twelve.
// The last case drops the final tile or (when there are segments) the final segment.
// *tile_count and *segment_count are updated; the arrays must hold one spare segment.
void tso_fabricate(void *engine, FabTile *tiles, std::uint64_t *tile_count,
                   FabSegment *segments, std::uint64_t *segment_count, std::uint64_t *file_bytes) {
    auto &rng = *static_cast<std::mt19937_64 *>(engine);
    FabTile &tile = tiles[rng() % *tile_count];
    FabSegment *segment = nullptr;
    if (*segment_count == 0) {
        segments[0] = FabSegment{};
        *segment_count = 1;
        segment = &segments[0];
    } else {
        segment = &segments[rng() % *segment_count];
    }
    switch (rng() % 12) {
    case 0: tile.mode = static_cast<std::uint32_t>(rng() % 4); break;
    case 1: tile.width = static_cast<std::uint16_t>(nudge(tile.width, rng, 1)); break;
    case 2: tile.height = static_cast<std::uint16_t>(nudge(tile.height, rng, 1)); break;
    case 3: tile.offset = nudge(tile.offset, rng, 4); break;
    case 4: tile.length = nudge(tile.length, rng, 4); break;
    case 5: tile.first_segment = nudge(tile.first_segment, rng, 1); break;
    case 6: segment->seed = static_cast<std::uint32_t>(nudge(segment->seed, rng, 1)); break;
    case 7: segment->bit_width = static_cast<std::uint32_t>(rng() % 40); break;
    case 8: segment->payload_offset = nudge(segment->payload_offset, rng, 4); break;
    case 9: segment->payload_bytes = nudge(segment->payload_bytes, rng, 4); break;
    case 10: *file_bytes = nudge(*file_bytes, rng, 4); break;
    default:
        if (rng() % 2 == 0) {
            --*tile_count;
        } else if (*segment_count != 0) {
            --*segment_count;
        }
        break;
    }
}

// harness.h:227-290: rebuilds the mutated .tsc file described by one mutation-corpus input.
// Returns 0 and the file in out (capacity cap) or a nonzero code when the corpus input does not
// describe a valid starting image or the file does not fit.
int tso_mutation_build(const std::uint8_t *data, std::uint64_t size, std::uint8_t *out,
                       std::uint64_t cap, std::uint64_t *out_size) {
    Reader in{data, static_cast<std::size_t>(size)};
    const auto config = in.take(1);
    const std::uint32_t type = config % 2 == 0 ? TSO_UINT16 : TSO_FLOAT32;
    const auto width = 1 + static_cast<std::uint32_t>(in.take(2) % 300);
    const auto height = 1 + static_cast<std::uint32_t>(in.take(2) % 160);
    const auto *shape = kShapes[config / 2 % 3];
    const auto pattern = static_cast<std::uint32_t>(in.take(1));
    const auto seed = in.take(4);
    const std::uint64_t s = type == TSO_UINT16 ? 2 : 4;
    const std::uint64_t row = width * s;
    std::vector<std::uint8_t> pixels(static_cast<std::size_t>(row * height));
    fill(type, width, height, row, pattern, seed, pixels.data());
    std::uint64_t bound = 0, written = 0;
    if (tso_compress_bound(type, width, height, shape[0], shape[1], &bound) != TSO_SUCCESS) {
        return 1;
    }
    std::vector<std::uint8_t> file(static_cast<std::size_t>(bound));
    if (tso_compress(pixels.data(), type, width, height, row, pixels.size(), shape[0], shape[1],
                     file.data(), bound, &written) != TSO_SUCCESS) {
        return 2;
    }
    file.resize(static_cast<std::size_t>(written));
    tso_layout layout{};
    if (tso_parse_layout(file.data(), file.size(), nullptr, &layout) != TSO_SUCCESS) return 3;
    std::vector<tso_tile> tiles(layout.tile_count);
    std::vector<tso_segment> segments(layout.segment_count + 1);
    if (tso_parse_fill(file.data(), file.size(), &layout, tiles.data(), segments.data()) !=
        TSO_SUCCESS) {
        return 3;
    }
    const auto payload = tiles[0].offset;
    for (int command = 0; command < 8 && !in.empty(); ++command) {
        const auto kind = in.take(1) % 6;
        const auto field = in.take(1);
        const auto target = in.take(2);
        const auto value = in.take(8);
        const auto index = target % tiles.size();
        const auto &t = tiles[static_cast<std::size_t>(index)];
        switch (kind) {
        case 0:
            change(file, 0, kHeader[field % 16], value);
            break;
        case 1:
            change(file, 64 + 32 * index, kEntry[field % 7], value);
            break;
        case 2:
            if (t.mode == TSO_PREDICT) {
                const auto &g = segments[static_cast<std::size_t>(t.first_segment +
                                                                  field % t.height)];
                change(file, t.offset + g.payload_offset - 8, kSegment[target % 3], value);
            }
            break;
        case 3:
            if (file.size() > payload) {
                file[static_cast<std::size_t>(payload + value % (file.size() - payload))] ^=
                    static_cast<std::uint8_t>(field | 1);
            }
            break;
        case 4:
            splice(file, tiles.size(), index, field, value);
            break;
        default:
            if (field % 2 == 0) {
                file.resize(static_cast<std::size_t>(value % (file.size() + 1)));
            } else {
                file.resize(file.size() + 1 + field % 8, static_cast<std::uint8_t>(value));
            }
            break;
        }
    }
    if (file.size() > cap) return 4;
    if (!file.empty()) std::memcpy(out, file.data(), file.size());
    *out_size = file.size();
    return 0;
}

} // extern "C"
