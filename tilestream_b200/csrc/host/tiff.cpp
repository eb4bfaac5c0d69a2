// TIFF import and export of include/tilestream/tiff.h, without libtiff.
//
// The container is the TIFF 6.0 one: an 8-byte header (byte order, 42, offset of the first
// image file directory), directories of 12-byte entries (tag, field type, count, value or
// offset) and the image as strips or tiles. BigTIFF (version 43) widens the header to 16 bytes,
// entries to 20 bytes and counts and offsets to 64 bits. Deflate strips and tiles are zlib
// streams (compression 8; 32946 is the older code for the same). Predictor 2 differences the
// samples along each row of a strip or tile; predictor 3 (floating point) splits the bytes of
// each row into planes, most significant first, and differences them byte by byte.
//
// Checks and their statuses follow the reference adapter (src/io/tiff.cpp:41-60 layout and
// limits, 62-105 tags, 107-186 tile and strip geometry, 205-236 write options, 240-343 entry
// points and the removal of a partly written file).
#include <tilestream/tiff.h>

#include "checked.h"

#include <zlib.h>

#include <sys/types.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

namespace tilestream::io {
namespace {

static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__,
              "samples are converted to and from little-endian host order");

// Tags.
constexpr std::uint16_t kImageWidth = 256, kImageLength = 257, kBitsPerSample = 258,
                        kCompression = 259, kPhotometric = 262, kStripOffsets = 273,
                        kOrientation = 274, kSamplesPerPixel = 277, kRowsPerStrip = 278,
                        kStripByteCounts = 279, kPlanarConfig = 284, kPredictor = 317,
                        kTileWidth = 322, kTileLength = 323, kTileOffsets = 324,
                        kTileByteCounts = 325, kSampleFormat = 339;
// Field types.
constexpr std::uint16_t kByte = 1, kShort = 3, kLong = 4, kIfd = 13, kLong8 = 16, kIfd8 = 18;
// Compression codes.
constexpr std::uint64_t kNone = 1, kDeflate = 8, kDeflateOld = 32946;

unsigned type_bytes(std::uint16_t type) {
    switch (type) {
    case kByte: return 1;
    case kShort: return 2;
    case kLong:
    case kIfd: return 4;
    case kLong8:
    case kIfd8: return 8;
    default: return 0; // not an integer field
    }
}

struct CloseFile {
    void operator()(std::FILE *f) const { std::fclose(f); }
};
using File = std::unique_ptr<std::FILE, CloseFile>;

// ---- reading ---------------------------------------------------------------------------

class Input {
  public:
    bool open(const char *path) {
        file_.reset(std::fopen(path, "rb"));
        if (!file_ || fseeko(file_.get(), 0, SEEK_END) != 0) return false;
        const off_t end = ftello(file_.get());
        if (end < 0) return false;
        size_ = static_cast<std::uint64_t>(end);
        return true;
    }
    // False when [offset, offset + bytes) is not inside the file or the read fails.
    bool read(std::uint64_t offset, std::uint64_t bytes, void *out) {
        if (offset > size_ || bytes > size_ - offset) return false;
        if (bytes == 0) return true;
        return fseeko(file_.get(), static_cast<off_t>(offset), SEEK_SET) == 0 &&
               std::fread(out, 1, static_cast<std::size_t>(bytes), file_.get()) == bytes;
    }
    std::uint64_t size() const { return size_; }

  private:
    File file_;
    std::uint64_t size_ = 0;
};

struct Entry {
    std::uint16_t type = 0;
    std::uint64_t count = 0;
    std::uint8_t field[8] = {}; // the value, or the offset of the values
};

// The header and the one image file directory of a file.
class Directory {
  public:
    bool big_endian() const { return big_endian_; }

    Status load(Input &in) {
        std::uint8_t head[16] = {};
        if (!in.read(0, 8, head)) return Status::io_error;
        if (head[0] == 'I' && head[1] == 'I') {
            big_endian_ = false;
        } else if (head[0] == 'M' && head[1] == 'M') {
            big_endian_ = true;
        } else {
            return Status::io_error; // not a TIFF file
        }
        const std::uint64_t version = get(head + 2, 2);
        std::uint64_t first = 0;
        if (version == 42) {
            first = get(head + 4, 4);
        } else if (version == 43) {
            if (!in.read(0, 16, head) || get(head + 4, 2) != 8 || get(head + 6, 2) != 0) {
                return Status::io_error;
            }
            bigtiff_ = true;
            first = get(head + 8, 8);
        } else {
            return Status::io_error;
        }
        const unsigned count_bytes = bigtiff_ ? 8 : 2, entry_bytes = bigtiff_ ? 20 : 12,
                       next_bytes = bigtiff_ ? 8 : 4;
        std::uint8_t raw[8] = {};
        if (first == 0 || !in.read(first, count_bytes, raw)) return Status::io_error;
        const std::uint64_t n = get(raw, count_bytes);
        const std::uint64_t room = in.size() - first - count_bytes;
        if (n == 0 || n > 65535 || n * entry_bytes + next_bytes > room) return Status::io_error;
        std::vector<std::uint8_t> block(static_cast<std::size_t>(n * entry_bytes + next_bytes));
        if (!in.read(first + count_bytes, block.size(), block.data())) return Status::io_error;
        for (std::uint64_t i = 0; i < n; ++i) {
            const std::uint8_t *e = block.data() + i * entry_bytes;
            Entry entry;
            const auto tag = static_cast<std::uint16_t>(get(e, 2));
            entry.type = static_cast<std::uint16_t>(get(e + 2, 2));
            entry.count = get(e + 4, bigtiff_ ? 8 : 4);
            std::memcpy(entry.field, e + (bigtiff_ ? 12 : 8), bigtiff_ ? 8 : 4);
            entries_.emplace(tag, entry); // a repeated tag keeps its first entry
        }
        // A second directory: one image per file only.
        if (get(block.data() + n * entry_bytes, next_bytes) != 0) return Status::unsupported_format;
        return Status::success;
    }

    bool has(std::uint16_t tag) const { return entries_.count(tag) != 0; }

    // The integer values of a field.
    Status values(Input &in, std::uint16_t tag, std::vector<std::uint64_t> &out) const {
        const auto it = entries_.find(tag);
        if (it == entries_.end()) return Status::unsupported_format;
        const Entry &e = it->second;
        const unsigned size = type_bytes(e.type);
        if (size == 0 || e.count == 0) return Status::unsupported_format;
        if (e.count > in.size()) return Status::io_error; // more values than the file holds
        const std::uint64_t bytes = e.count * size;
        std::vector<std::uint8_t> raw;
        const std::uint8_t *p = e.field;
        if (bytes > (bigtiff_ ? 8u : 4u)) {
            raw.resize(static_cast<std::size_t>(bytes));
            if (!in.read(get(e.field, bigtiff_ ? 8 : 4), bytes, raw.data())) {
                return Status::io_error;
            }
            p = raw.data();
        }
        out.resize(static_cast<std::size_t>(e.count));
        for (std::uint64_t i = 0; i < e.count; ++i) {
            out[static_cast<std::size_t>(i)] = get(p + i * size, size);
        }
        return Status::success;
    }

    // The first value of a field, or `fallback` when the field is absent.
    Status scalar(Input &in, std::uint16_t tag, std::uint64_t fallback, std::uint64_t &out) const {
        if (!has(tag)) {
            out = fallback;
            return Status::success;
        }
        std::vector<std::uint64_t> v;
        const Status st = values(in, tag, v);
        if (st == Status::success) out = v[0];
        return st;
    }

  private:
    std::uint64_t get(const std::uint8_t *p, unsigned n) const {
        std::uint64_t v = 0;
        for (unsigned i = 0; i < n; ++i) {
            v |= std::uint64_t{p[big_endian_ ? n - 1 - i : i]} << (8 * i);
        }
        return v;
    }

    bool big_endian_ = false, bigtiff_ = false;
    std::map<std::uint16_t, Entry> entries_;
};

// How the pixels of one file are stored.
struct Layout {
    ImageSpec image;
    std::uint64_t sample = 0, row_bytes = 0, total = 0;
    bool deflate = false, big_endian = false;
    std::uint64_t predictor = 1;
    bool tiled = false;
    std::uint64_t block_width = 0, block_height = 0; // tile, or image width x rows per strip
    std::vector<std::uint64_t> offsets, counts;
};

Status read_tags(Input &in, const Directory &dir, const TiffReadLimits &limits, Layout &L) {
    std::uint64_t width = 0, height = 0, samples = 0, bits = 0, format = 0, planar = 0,
                  orientation = 0, photometric = 0, compression = 0, predictor = 0;
    if (!dir.has(kImageWidth) || !dir.has(kImageLength)) return Status::unsupported_format;
    const struct {
        std::uint16_t tag;
        std::uint64_t fallback;
        std::uint64_t *out;
    } fields[] = {{kImageWidth, 0, &width},         {kImageLength, 0, &height},
                  {kSamplesPerPixel, 1, &samples},  {kBitsPerSample, 1, &bits},
                  {kSampleFormat, 1, &format},      {kPlanarConfig, 1, &planar},
                  {kOrientation, 1, &orientation},  {kPhotometric, 1, &photometric},
                  {kCompression, kNone, &compression}, {kPredictor, 1, &predictor}};
    for (const auto &f : fields) {
        const Status st = dir.scalar(in, f.tag, f.fallback, *f.out);
        if (st != Status::success) return st;
    }
    if (samples != 1 || planar != 1 || orientation != 1 || photometric != 1) {
        return Status::unsupported_format;
    }
    if (bits == 16 && format == 1) {
        L.image.type = PixelType::uint16;
    } else if (bits == 32 && format == 3) {
        L.image.type = PixelType::float32;
    } else {
        return Status::unsupported_format;
    }
    if (width > UINT32_MAX || height > UINT32_MAX) return Status::unsupported_format;
    L.image.width = static_cast<std::uint32_t>(width);
    L.image.height = static_cast<std::uint32_t>(height);
    if (width == 0 || height == 0) return Status::unsupported_format;
    if (width > limits.max_width || height > limits.max_height) return Status::resource_limit;
    L.sample = L.image.type == PixelType::uint16 ? 2 : 4;
    if (!host::mul(width, L.sample, L.row_bytes) || !host::mul(L.row_bytes, height, L.total)) {
        return Status::size_overflow;
    }
    if (L.total > limits.max_decoded_bytes) return Status::resource_limit;
    if (compression == kNone) {
        L.deflate = false;
        L.predictor = 1; // a predictor applies to compressed data only
    } else if (compression == kDeflate || compression == kDeflateOld) {
        L.deflate = true;
        if (predictor != 1 && predictor != 2 && !(predictor == 3 && format == 3)) {
            return Status::unsupported_format;
        }
        L.predictor = predictor;
    } else {
        return Status::unsupported_format;
    }
    L.big_endian = dir.big_endian();
    return Status::success;
}

Status read_geometry(Input &in, const Directory &dir, Layout &L) {
    std::uint64_t blocks = 0;
    L.tiled = dir.has(kTileWidth);
    if (L.tiled) {
        Status st = dir.scalar(in, kTileWidth, 0, L.block_width);
        if (st == Status::success) st = dir.scalar(in, kTileLength, 0, L.block_height);
        if (st != Status::success) return st;
        if (!dir.has(kTileLength) || L.block_width == 0 || L.block_height == 0 ||
            L.block_width > UINT32_MAX || L.block_height > UINT32_MAX) {
            return Status::unsupported_format;
        }
        std::uint64_t bytes = 0;
        if (!host::mul(L.block_width, L.block_height, bytes) ||
            !host::mul(bytes, L.sample, bytes)) {
            return Status::size_overflow;
        }
        const std::uint64_t across = host::ceil_div(L.image.width, L.block_width);
        const std::uint64_t down = host::ceil_div(L.image.height, L.block_height);
        if (!host::mul(across, down, blocks) || blocks > UINT32_MAX) return Status::size_overflow;
    } else {
        std::uint64_t rows = 0;
        const Status st = dir.scalar(in, kRowsPerStrip, UINT32_MAX, rows);
        if (st != Status::success) return st;
        if (rows == 0) return Status::unsupported_format;
        L.block_width = L.image.width;
        L.block_height = std::min<std::uint64_t>(rows, L.image.height);
        std::uint64_t bytes = 0;
        if (!host::mul(L.row_bytes, L.block_height, bytes)) return Status::size_overflow;
        blocks = host::ceil_div(L.image.height, L.block_height);
    }
    const std::uint16_t offsets_tag =
        L.tiled && dir.has(kTileOffsets) ? kTileOffsets : kStripOffsets;
    const std::uint16_t counts_tag =
        L.tiled && dir.has(kTileByteCounts) ? kTileByteCounts : kStripByteCounts;
    Status st = dir.values(in, offsets_tag, L.offsets);
    if (st == Status::success) st = dir.values(in, counts_tag, L.counts);
    if (st != Status::success) return st;
    if (L.offsets.size() != blocks || L.counts.size() != blocks) return Status::unsupported_format;
    return Status::success;
}

// Inflates `bytes` of zlib stream into exactly `expected` bytes; false when it holds fewer or
// is not a valid stream.
bool inflate_block(const std::uint8_t *src, std::uint64_t bytes, std::uint8_t *out,
                   std::uint64_t expected) {
    z_stream z{};
    if (inflateInit(&z) != Z_OK) return false;
    z.next_in = const_cast<Bytef *>(src);
    std::uint64_t in_left = bytes, out_done = 0;
    while (out_done < expected) {
        if (z.avail_in == 0 && in_left != 0) {
            // zlib advances next_in itself; only the count of the next chunk is set here.
            z.avail_in = static_cast<uInt>(std::min<std::uint64_t>(in_left, 1u << 30));
            in_left -= z.avail_in;
        }
        z.next_out = out + out_done;
        z.avail_out = static_cast<uInt>(std::min<std::uint64_t>(expected - out_done, 1u << 30));
        const uInt before = z.avail_out;
        const int rc = inflate(&z, Z_NO_FLUSH);
        out_done += before - z.avail_out;
        if (rc == Z_STREAM_END || (rc != Z_OK && rc != Z_BUF_ERROR)) break;
        if (rc == Z_BUF_ERROR && z.avail_in == 0 && in_left == 0) break; // input ran out
    }
    inflateEnd(&z);
    return out_done == expected;
}

// The stored bytes of one block (strip or tile) of `rows` rows of `width` samples, decoded
// into host-order samples at `out`.
Status read_block(Input &in, const Layout &L, std::uint64_t index, std::uint64_t width,
                  std::uint64_t rows, std::uint8_t *out, std::vector<std::uint8_t> &scratch) {
    const std::uint64_t row = width * L.sample, expected = row * rows;
    const std::uint64_t offset = L.offsets[static_cast<std::size_t>(index)];
    const std::uint64_t stored = L.counts[static_cast<std::size_t>(index)];
    // The whole stored block must lie in the file, even where fewer bytes are needed.
    if (offset > in.size() || stored > in.size() - offset) return Status::io_error;
    if (!L.deflate) {
        if (stored < expected || !in.read(offset, expected, out)) return Status::io_error;
    } else {
        scratch.resize(static_cast<std::size_t>(stored));
        if (!in.read(offset, stored, scratch.data()) ||
            !inflate_block(scratch.data(), stored, out, expected)) {
            return Status::io_error;
        }
    }
    if (L.predictor == 3) {
        // Byte planes (most significant first) differenced along the row.
        std::vector<std::uint8_t> planes(static_cast<std::size_t>(row));
        for (std::uint64_t r = 0; r < rows; ++r) {
            std::uint8_t *p = out + r * row;
            for (std::uint64_t i = 1; i < row; ++i) p[i] = static_cast<std::uint8_t>(p[i] + p[i - 1]);
            std::memcpy(planes.data(), p, static_cast<std::size_t>(row));
            for (std::uint64_t x = 0; x < width; ++x) {
                for (std::uint64_t b = 0; b < L.sample; ++b) {
                    p[x * L.sample + b] = planes[(L.sample - 1 - b) * width + x];
                }
            }
        }
        return Status::success;
    }
    if (L.big_endian) {
        for (std::uint64_t i = 0; i < expected; i += L.sample) {
            std::reverse(out + i, out + i + L.sample);
        }
    }
    if (L.predictor == 2) {
        for (std::uint64_t r = 0; r < rows; ++r) {
            std::uint8_t *p = out + r * row;
            if (L.sample == 2) {
                for (std::uint64_t x = 1; x < width; ++x) {
                    std::uint16_t a, b;
                    std::memcpy(&a, p + (x - 1) * 2, 2);
                    std::memcpy(&b, p + x * 2, 2);
                    b = static_cast<std::uint16_t>(a + b);
                    std::memcpy(p + x * 2, &b, 2);
                }
            } else {
                for (std::uint64_t x = 1; x < width; ++x) {
                    std::uint32_t a, b;
                    std::memcpy(&a, p + (x - 1) * 4, 4);
                    std::memcpy(&b, p + x * 4, 4);
                    b += a;
                    std::memcpy(p + x * 4, &b, 4);
                }
            }
        }
    }
    return Status::success;
}

Status read_pixels(Input &in, const Layout &L, TiffImage &image) {
    std::vector<std::uint8_t> scratch;
    const std::uint64_t w = L.image.width, h = L.image.height;
    if (!L.tiled) {
        // Strips hold whole rows: each is decoded in place.
        for (std::uint64_t s = 0; s * L.block_height < h; ++s) {
            const std::uint64_t y = s * L.block_height;
            const std::uint64_t rows = std::min(L.block_height, h - y);
            const Status st = read_block(in, L, s, w, rows, image.pixels.data() + y * L.row_bytes,
                                         scratch);
            if (st != Status::success) return st;
        }
        return Status::success;
    }
    std::vector<std::uint8_t> tile(
        static_cast<std::size_t>(L.block_width * L.block_height * L.sample));
    for (std::uint64_t y = 0, t = 0; y < h; y += L.block_height) {
        for (std::uint64_t x = 0; x < w; x += L.block_width, ++t) {
            const Status st = read_block(in, L, t, L.block_width, L.block_height, tile.data(),
                                         scratch);
            if (st != Status::success) return st;
            const std::uint64_t cw = std::min(L.block_width, w - x) * L.sample;
            const std::uint64_t ch = std::min(L.block_height, h - y);
            for (std::uint64_t r = 0; r < ch; ++r) {
                std::memcpy(image.pixels.data() + (y + r) * L.row_bytes + x * L.sample,
                            tile.data() + r * L.block_width * L.sample,
                            static_cast<std::size_t>(cw));
            }
        }
    }
    return Status::success;
}

// ---- writing ---------------------------------------------------------------------------

// An output file that is removed unless it was completed.
class Output {
  public:
    explicit Output(const char *path) : path_(path), file_(std::fopen(path, "wb")) {}
    ~Output() {
        if (file_ != nullptr && !done_) {
            std::fclose(file_);
            std::remove(path_.c_str());
        }
    }
    bool is_open() const { return file_ != nullptr; }
    std::uint64_t position() const { return position_; }
    bool write(const void *data, std::uint64_t bytes) {
        if (bytes != 0 && std::fwrite(data, 1, static_cast<std::size_t>(bytes), file_) != bytes) {
            return false;
        }
        position_ += bytes;
        return true;
    }
    bool pad_to_even() {
        static const std::uint8_t zero = 0;
        return position_ % 2 == 0 || write(&zero, 1);
    }
    bool write_at(std::uint64_t offset, const void *data, std::uint64_t bytes) {
        return fseeko(file_, static_cast<off_t>(offset), SEEK_SET) == 0 &&
               std::fwrite(data, 1, static_cast<std::size_t>(bytes), file_) == bytes;
    }
    bool finish() {
        const bool ok = std::fflush(file_) == 0;
        const bool closed = std::fclose(file_) == 0;
        done_ = ok && closed;
        if (!done_) std::remove(path_.c_str());
        file_ = nullptr;
        return done_;
    }

  private:
    std::string path_;
    std::FILE *file_ = nullptr;
    std::uint64_t position_ = 0;
    bool done_ = false;
};

struct OutEntry {
    std::uint16_t tag, type;
    std::uint64_t count;
    std::uint64_t field; // little-endian value bytes, or the offset of the values
};

Status validate(ConstImageView image, const TiffWriteOptions &options) {
    const Status st = host::view_ok(image);
    if (st != Status::success) return st;
    if (options.compression != TiffCompression::none &&
        options.compression != TiffCompression::deflate) {
        return Status::invalid_argument;
    }
    if (options.tile_width == 0 || options.tile_height == 0 || options.tile_width % 16 != 0 ||
        options.tile_height % 16 != 0) {
        return Status::invalid_argument;
    }
    if (options.horizontal_predictor && (image.image.type != PixelType::uint16 ||
                                         options.compression != TiffCompression::deflate)) {
        return Status::invalid_argument;
    }
    if (options.compression == TiffCompression::deflate &&
        (options.deflate_level < 1 || options.deflate_level > 9)) {
        return Status::invalid_argument;
    }
    return Status::success;
}

Status write_file(const char *path, ConstImageView image, const TiffWriteOptions &o,
                  std::uint64_t tile_bytes, std::uint64_t across, std::uint64_t down) {
    Output out(path);
    if (!out.is_open()) return Status::io_error;
    const bool big = o.bigtiff, deflate = o.compression == TiffCompression::deflate;
    const std::uint64_t sample = image.image.type == PixelType::uint16 ? 2 : 4;
    const std::uint64_t count = across * down;
    // Header; the directory offset is filled in at the end.
    std::uint8_t head[16] = {'I', 'I'};
    host::put_le(head + 2, big ? 43 : 42, 2);
    if (big) host::put_le(head + 4, 8, 2);
    if (!out.write(head, big ? 16 : 8)) return Status::io_error;

    std::vector<std::uint64_t> offsets(static_cast<std::size_t>(count)),
        sizes(static_cast<std::size_t>(count));
    std::vector<std::uint8_t> tile(static_cast<std::size_t>(tile_bytes)), packed;
    if (deflate) packed.resize(static_cast<std::size_t>(compressBound(static_cast<uLong>(tile_bytes))));
    const auto *src = static_cast<const std::uint8_t *>(image.data);
    const std::uint64_t row = std::uint64_t{o.tile_width} * sample;
    for (std::uint64_t ty = 0, t = 0; ty < down; ++ty) {
        for (std::uint64_t tx = 0; tx < across; ++tx, ++t) {
            const std::uint64_t x = tx * o.tile_width, y = ty * o.tile_height;
            const std::uint64_t cw = std::min<std::uint64_t>(o.tile_width, image.image.width - x);
            const std::uint64_t ch = std::min<std::uint64_t>(o.tile_height, image.image.height - y);
            std::fill(tile.begin(), tile.end(), 0);
            for (std::uint64_t r = 0; r < ch; ++r) {
                std::memcpy(tile.data() + r * row, src + (y + r) * image.pitch_bytes + x * sample,
                            static_cast<std::size_t>(cw * sample));
            }
            if (o.horizontal_predictor) {
                for (std::uint64_t r = 0; r < o.tile_height; ++r) {
                    std::uint8_t *p = tile.data() + r * row;
                    for (std::uint64_t i = o.tile_width; i-- > 1;) {
                        std::uint16_t a, b;
                        std::memcpy(&a, p + (i - 1) * 2, 2);
                        std::memcpy(&b, p + i * 2, 2);
                        b = static_cast<std::uint16_t>(b - a);
                        std::memcpy(p + i * 2, &b, 2);
                    }
                }
            }
            const std::uint8_t *data = tile.data();
            std::uint64_t bytes = tile_bytes;
            if (deflate) {
                uLongf packed_bytes = static_cast<uLongf>(packed.size());
                if (compress2(packed.data(), &packed_bytes, tile.data(),
                              static_cast<uLong>(tile_bytes),
                              static_cast<int>(o.deflate_level)) != Z_OK) {
                    return Status::io_error;
                }
                data = packed.data();
                bytes = packed_bytes;
            }
            offsets[static_cast<std::size_t>(t)] = out.position();
            sizes[static_cast<std::size_t>(t)] = bytes;
            if (!out.write(data, bytes)) return Status::io_error;
        }
    }
    // Classic TIFF addresses 4 GiB.
    if (!big && out.position() > UINT32_MAX) return Status::io_error;

    // Offset and byte-count arrays that do not fit in their entries.
    const unsigned width = big ? 8 : 4; // bytes per value and per entry field
    const std::uint16_t array_type = big ? kLong8 : kLong;
    auto place = [&](const std::vector<std::uint64_t> &v, std::uint64_t &field) {
        if (v.size() * width <= width) {
            field = v[0];
            return true;
        }
        if (!out.pad_to_even()) return false;
        field = out.position();
        std::vector<std::uint8_t> raw(v.size() * width);
        for (std::size_t i = 0; i < v.size(); ++i) host::put_le(raw.data() + i * width, v[i], width);
        return out.write(raw.data(), raw.size());
    };
    std::uint64_t offsets_field = 0, sizes_field = 0;
    if (!place(offsets, offsets_field) || !place(sizes, sizes_field)) return Status::io_error;

    std::vector<OutEntry> entries = {
        {kImageWidth, kLong, 1, image.image.width},
        {kImageLength, kLong, 1, image.image.height},
        {kBitsPerSample, kShort, 1, sample * 8},
        {kCompression, kShort, 1, deflate ? kDeflate : kNone},
        {kPhotometric, kShort, 1, 1},  // min-is-black
        {kOrientation, kShort, 1, 1},  // top-left
        {kSamplesPerPixel, kShort, 1, 1},
        {kPlanarConfig, kShort, 1, 1}, // contiguous
        {kTileWidth, kLong, 1, o.tile_width},
        {kTileLength, kLong, 1, o.tile_height},
        {kTileOffsets, array_type, count, offsets_field},
        {kTileByteCounts, array_type, count, sizes_field},
        {kSampleFormat, kShort, 1, image.image.type == PixelType::uint16 ? 1u : 3u},
    };
    if (deflate) entries.push_back({kPredictor, kShort, 1, o.horizontal_predictor ? 2u : 1u});
    std::sort(entries.begin(), entries.end(),
              [](const OutEntry &a, const OutEntry &b) { return a.tag < b.tag; });
    if (!out.pad_to_even()) return Status::io_error;
    const std::uint64_t directory = out.position();
    const unsigned entry_bytes = big ? 20 : 12, count_bytes = big ? 8 : 2;
    std::vector<std::uint8_t> block(count_bytes + entries.size() * entry_bytes + width, 0);
    if (!big && directory + block.size() > UINT32_MAX) return Status::io_error;
    host::put_le(block.data(), entries.size(), count_bytes);
    for (std::size_t i = 0; i < entries.size(); ++i) {
        std::uint8_t *e = block.data() + count_bytes + i * entry_bytes;
        host::put_le(e, entries[i].tag, 2);
        host::put_le(e + 2, entries[i].type, 2);
        host::put_le(e + 4, entries[i].count, big ? 8 : 4);
        host::put_le(e + (big ? 12 : 8), entries[i].field, width);
    }
    if (!out.write(block.data(), block.size())) return Status::io_error;
    std::uint8_t at[8];
    host::put_le(at, directory, width);
    if (!out.write_at(big ? 8 : 4, at, width) || !out.finish()) return Status::io_error;
    return Status::success;
}

} // namespace

Status read_tiff(const char *path, TiffImage &image, const TiffReadLimits &limits) noexcept {
    if (path == nullptr || limits.max_width == 0 || limits.max_height == 0 ||
        limits.max_decoded_bytes > max_bytes) {
        return Status::invalid_argument;
    }
    try {
        Input in;
        if (!in.open(path)) return Status::io_error;
        Directory dir;
        Status st = dir.load(in);
        Layout layout;
        if (st == Status::success) st = read_tags(in, dir, limits, layout);
        if (st == Status::success) st = read_geometry(in, dir, layout);
        if (st != Status::success) return st;
        TiffImage decoded;
        decoded.image = layout.image;
        decoded.pitch_bytes = layout.row_bytes;
        decoded.pixels.resize(static_cast<std::size_t>(layout.total));
        st = read_pixels(in, layout, decoded);
        if (st != Status::success) return st;
        image = std::move(decoded);
        return Status::success;
    } catch (const std::bad_alloc &) {
        return Status::resource_limit;
    } catch (const std::length_error &) {
        return Status::resource_limit;
    }
}

Status write_tiff(const char *path, ConstImageView image,
                  const TiffWriteOptions &options) noexcept {
    if (path == nullptr) return Status::invalid_argument;
    const Status st = validate(image, options);
    if (st != Status::success) return st;
    const std::uint64_t sample = image.image.type == PixelType::uint16 ? 2 : 4;
    std::uint64_t tile_bytes = 0, count = 0;
    if (!host::mul(options.tile_width, options.tile_height, tile_bytes) ||
        !host::mul(tile_bytes, sample, tile_bytes)) {
        return Status::size_overflow;
    }
    const std::uint64_t across = host::ceil_div(image.image.width, options.tile_width);
    const std::uint64_t down = host::ceil_div(image.image.height, options.tile_height);
    if (!host::mul(across, down, count) || count > UINT32_MAX) return Status::size_overflow;
    // A failed write_file has removed its partial file already.
    try {
        return write_file(path, image, options, tile_bytes, across, down);
    } catch (const std::bad_alloc &) {
        return Status::resource_limit;
    } catch (const std::length_error &) {
        return Status::resource_limit;
    }
}

} // namespace tilestream::io
