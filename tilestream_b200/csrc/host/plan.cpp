// prepare_batch, check_execution and the five executors of include/tilestream/cuda.h.
//
// Host validation covers the same conditions, in the same order and with the same statuses, as
// the reference planner (src/cuda/plan.cpp:128-465, 627-711), so error behaviour is a drop-in.
// What the plan builds is different: instead of DeviceImage/DeviceTile/DeviceSegment tables
// split into 4096-tile windows with a binary search per block, every execution is one
// persistent launch over a flat queue of self-contained tasks (tsk_decode_task, one per tile
// to decode, 64 bytes), plus a 16-byte-aligned slot of row starts per predictive tile that the
// kernel stages with the payload. The WorkspaceSpec reported to callers is still the
// reference's per-window bound, so workspace_size() callers allocate what they always did.
#include "plan.h"

#include <tilestream/batch.h>

#include <map>
#include <mutex>
#include <string>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <stdexcept>
#include <utility>

namespace tilestream::cuda {
namespace detail {

constexpr std::uint32_t kWindowTiles = 4096; // the reference's window bound (plan.h:14)

// One sweep over every non-empty range in order of its first byte. A range overlaps an earlier
// one exactly when it starts before that one ends, so it is enough to carry two high-water
// marks: the furthest end of any earlier range and of any earlier writable range. The same
// sweep builds the coalesced union that disjoint() searches.
bool RangeSet::assign(std::vector<Range> writable, std::vector<Range> readable) {
    struct Tagged {
        Range range;
        bool writes;
    };
    std::vector<Tagged> all;
    all.reserve(writable.size() + readable.size());
    for (const Range &r : writable) {
        if (r.end != r.begin) all.push_back({r, true});
    }
    for (const Range &r : readable) {
        if (r.end != r.begin) all.push_back({r, false});
    }
    std::sort(all.begin(), all.end(),
              [](const Tagged &a, const Tagged &b) { return a.range.begin < b.range.begin; });
    std::uintptr_t any_end = 0, written_end = 0;
    std::vector<Range> spans;
    for (const Tagged &t : all) {
        const bool clash = t.writes ? t.range.begin < any_end : t.range.begin < written_end;
        if (clash) {
            return false;
        }
        if (!spans.empty() && t.range.begin <= spans.back().end) {
            spans.back().end = std::max(spans.back().end, t.range.end);
        } else {
            spans.push_back(t.range);
        }
        any_end = std::max(any_end, t.range.end);
        if (t.writes) {
            written_end = std::max(written_end, t.range.end);
        }
    }
    spans_ = std::move(spans);
    return true;
}

bool RangeSet::disjoint(Range range) const noexcept {
    if (range.begin == range.end) {
        return true;
    }
    // The first span that ends after range.begin is the only candidate for an overlap.
    const auto it = std::upper_bound(spans_.begin(), spans_.end(), range.begin,
                                     [](std::uintptr_t at, const Range &s) { return at < s.end; });
    return it == spans_.end() || it->begin >= range.end;
}

PlanState::~PlanState() {
    // Executions must have finished (docs/api.md:71), so the free needs no ordering.
    if (storage != nullptr) {
        static_cast<void>(cuda_status(cudaFreeAsync(storage, cudaStreamPerThread)));
    }
}

void log_failure(const char *what, cudaError_t error) noexcept {
    static const bool enabled = std::getenv("TILESTREAM_DEBUG") != nullptr;
    if (enabled) {
        std::fprintf(stderr, "tilestream: %s failed: %s (%d)\n", what, cudaGetErrorName(error),
                     static_cast<int>(error));
    }
}

Status accessible(const void *data, int device, bool pageable) noexcept {
    cudaPointerAttributes a{};
    const cudaError_t e = cudaPointerGetAttributes(&a, data);
    if (e != cudaSuccess) {
        return cuda_failure("cudaPointerGetAttributes", e);
    }
    switch (a.type) {
    case cudaMemoryTypeDevice:
        return a.device == device ? Status::success : Status::invalid_argument;
    case cudaMemoryTypeManaged:
        return Status::success;
    case cudaMemoryTypeHost:
        return a.devicePointer == data ? Status::success : Status::invalid_argument;
    default:
        return pageable ? Status::success : Status::invalid_argument;
    }
}

Status stream_device(cudaStream_t stream, int device) noexcept {
    int current = 0, owner = 0;
    cudaError_t e = cudaGetDevice(&current);
    if (e != cudaSuccess) {
        return cuda_failure("cudaGetDevice", e);
    }
    // A stream that is being captured into a CUDA graph cannot be asked for its device
    // (cudaErrorStreamCaptureUnsupported); the capture then checks the current device only and
    // the launch itself rejects a stream of another device.
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(stream, &capture);
    if (e != cudaSuccess) {
        return cuda_failure("cudaStreamIsCapturing", e);
    }
    if (capture == cudaStreamCaptureStatusNone) {
        e = cudaStreamGetDevice(stream, &owner);
        if (e != cudaSuccess) {
            return cuda_failure("cudaStreamGetDevice", e);
        }
    } else {
        owner = current;
    }
    return current == device && owner == device ? Status::success : Status::invalid_argument;
}

namespace {

std::uint64_t tiles_across(const ImageSpec &im, TileShape t) noexcept {
    return host::ceil_div(im.width, t.width);
}
std::uint64_t tiles_down(const ImageSpec &im, TileShape t) noexcept {
    return host::ceil_div(im.height, t.height);
}

// Host-side draft of a plan: validated descriptors and the ranges/pointers to check.
struct Draft {
    PixelType type = PixelType::uint16;
    TileShape shape;
    std::vector<std::uint64_t> tiles_per_image; // for the reference window accounting
    std::vector<Range> writable, readable;
    std::vector<const void *> pointers;

    std::vector<tsk_decode_image> images;
    std::vector<tsk_decode_task> tasks;
    std::vector<tsk_row_start> rows;
    bool trusted = false;
    bool any_u16 = false, any_f32 = false, any_plain = false, any_calibrated = false;

    std::vector<tsk_encode_image> encode_images;
    std::uint64_t total_tiles = 0;

    std::vector<tsk_calib_image> calib_images;
    std::vector<tsk_calib_task> calib_tasks;
};

Status draft_compress(const BatchRequest &request, Draft &d) {
    d.type = request.items[0].input.image.type;
    d.shape = request.tile;
    for (std::uint64_t i = 0; i < request.count; ++i) {
        const BatchItem &item = request.items[i];
        Status st = host::view_ok(item.input);
        if (st != Status::success) {
            return st;
        }
        if (item.input.image.type != d.type) {
            return Status::invalid_argument;
        }
        std::uint64_t bound = 0;
        st = compress_bound(item.input.image, request.tile, bound);
        if (st != Status::success) {
            return st;
        }
        const MutableBytes &out = item.compressed_output;
        st = host::byte_range(out.data, out.size);
        if (st != Status::success) {
            return st;
        }
        if (out.data == nullptr || reinterpret_cast<std::uintptr_t>(out.data) % 4 != 0) {
            return Status::invalid_argument;
        }
        if (out.size < bound) {
            return Status::buffer_too_small;
        }
        tsk_encode_image e{};
        e.input = reinterpret_cast<std::uint64_t>(item.input.data);
        e.pitch = item.input.pitch_bytes;
        e.output = reinterpret_cast<std::uint64_t>(out.data);
        e.columns = tiles_across(item.input.image, request.tile);
        e.tile_count = e.columns * tiles_down(item.input.image, request.tile);
        e.first_tile = d.total_tiles;
        e.width = item.input.image.width;
        e.height = item.input.image.height;
        e.tile_width = request.tile.width;
        e.tile_height = request.tile.height;
        e.type = static_cast<std::uint32_t>(item.input.image.type);
        d.total_tiles += e.tile_count;
        d.encode_images.push_back(e);
        d.tiles_per_image.push_back(e.tile_count);
        d.readable.push_back(range_of(item.input.data, item.input.capacity_bytes));
        d.writable.push_back(range_of(out.data, out.size));
        d.pointers.push_back(item.input.data);
        d.pointers.push_back(out.data);
    }
    return Status::success;
}

// A map matches the output region exactly and is addressed in output coordinates.
Status check_parameter(const Parameter &p, const ImageSpec &region, Draft &d) {
    if (p.kind == ParameterKind::scalar) {
        return Status::success;
    }
    if (p.kind != ParameterKind::map) {
        return Status::invalid_argument;
    }
    const Status st = host::view_ok(p.map);
    if (st != Status::success) {
        return st;
    }
    if (p.map.image.type != PixelType::float32 || p.map.image.width != region.width ||
        p.map.image.height != region.height) {
        return Status::invalid_argument;
    }
    d.readable.push_back(range_of(p.map.data, p.map.capacity_bytes));
    d.pointers.push_back(p.map.data);
    return Status::success;
}

Status check_calibration(const Calibration &c, const ImageSpec &region, Draft &d) {
    const Status st = check_parameter(c.offset, region, d);
    return st != Status::success ? st : check_parameter(c.gain, region, d);
}

void set_parameters(const Calibration &c, std::uint64_t &offset_map, std::uint64_t &offset_pitch,
                    float &offset, std::uint64_t &gain_map, std::uint64_t &gain_pitch,
                    float &gain) {
    offset_map = c.offset.kind == ParameterKind::map
                     ? reinterpret_cast<std::uint64_t>(c.offset.map.data)
                     : 0;
    offset_pitch = c.offset.map.pitch_bytes;
    offset = c.offset.scalar;
    gain_map =
        c.gain.kind == ParameterKind::map ? reinterpret_cast<std::uint64_t>(c.gain.map.data) : 0;
    gain_pitch = c.gain.map.pitch_bytes;
    gain = c.gain.scalar;
}

Status draft_calibrate(const BatchRequest &request, Draft &d) {
    d.type = request.items[0].input.image.type;
    for (std::uint64_t i = 0; i < request.count; ++i) {
        const BatchItem &item = request.items[i];
        Status st = host::view_ok(item.input);
        if (st == Status::success) {
            st = host::view_ok(item.output);
        }
        if (st != Status::success) {
            return st;
        }
        if (item.input.image.type != d.type || item.output.image.type != PixelType::float32 ||
            item.output.image.width != item.input.image.width ||
            item.output.image.height != item.input.image.height) {
            return Status::invalid_argument;
        }
        st = check_calibration(item.calibration, item.output.image, d);
        if (st != Status::success) {
            return st;
        }
        tsk_calib_image c{};
        c.input = reinterpret_cast<std::uint64_t>(item.input.data);
        c.in_pitch = item.input.pitch_bytes;
        c.out = reinterpret_cast<std::uint64_t>(item.output.data);
        c.out_pitch = item.output.pitch_bytes;
        set_parameters(item.calibration, c.offset_map, c.offset_pitch, c.offset, c.gain_map,
                       c.gain_pitch, c.gain);
        c.width = item.input.image.width;
        c.height = item.input.image.height;
        c.type = static_cast<std::uint32_t>(item.input.image.type);
        const auto image = static_cast<std::uint32_t>(d.calib_images.size());
        // Chunks of about 16 Ki pixels keep every SM streaming on small and large images alike.
        // About 4 Ki pixels per task: enough work per task, and rounds fine enough that the
        // persistent grid ends evenly.
        const std::uint32_t chunk = std::max<std::uint32_t>(1, 4096 / c.width);
        for (std::uint32_t y = 0; y < c.height; y += chunk) {
            tsk_calib_task t{};
            t.image = image;
            t.y0 = y;
            t.rows = std::min(chunk, c.height - y);
            t.reserved = y == 0 ? 1u : 0u; // first chunk writes the result record
            d.calib_tasks.push_back(t);
        }
        d.calib_images.push_back(c);
        d.tiles_per_image.push_back(0);
        d.readable.push_back(range_of(item.input.data, item.input.capacity_bytes));
        d.writable.push_back(range_of(item.output.data, item.output.capacity_bytes));
        d.pointers.push_back(item.input.data);
        d.pointers.push_back(item.output.data);
    }
    return Status::success;
}

} // namespace

// Repeats the parser's structural checks that keep device reads inside the tile payload
// (reference plan.cpp:237-279).
Status check_tile(const ImageMetadata &m, std::uint64_t index) noexcept {
    const TileMetadata &t = m.tiles[static_cast<std::size_t>(index)];
    const std::uint64_t across = tiles_across(m.image, m.tile);
    const std::uint64_t x = index % across * m.tile.width;
    const std::uint64_t y = index / across * m.tile.height;
    const std::uint64_t w = std::min<std::uint64_t>(m.tile.width, m.image.width - x);
    const std::uint64_t h = std::min<std::uint64_t>(m.tile.height, m.image.height - y);
    const std::uint64_t s = m.image.type == PixelType::uint16 ? 2 : 4;
    const std::uint32_t max_bits = m.image.type == PixelType::uint16 ? 16 : 32;
    const std::uint64_t raw = (w * h * s + 3) / 4 * 4;
    if (t.width != w || t.height != h || t.offset % 4 != 0 || t.offset > m.file_bytes ||
        t.length > m.file_bytes - t.offset) {
        return Status::malformed_data;
    }
    switch (t.mode) {
    case TileMode::raw:
        return t.length == raw ? Status::success : Status::malformed_data;
    case TileMode::constant:
        return t.length == 4 ? Status::success : Status::malformed_data;
    case TileMode::predict_bitpack:
        break;
    default:
        return Status::malformed_data;
    }
    if (t.length > raw || t.first_segment > m.segments.size() ||
        h > m.segments.size() - t.first_segment) {
        return Status::malformed_data;
    }
    for (std::uint64_t r = 0; r < h; ++r) {
        const SegmentMetadata &g = m.segments[static_cast<std::size_t>(t.first_segment + r)];
        if (g.bit_width > max_bits || (m.image.type == PixelType::uint16 && g.seed > UINT16_MAX) ||
            g.payload_offset < format::segment_header_bytes || g.payload_offset % 4 != 0 ||
            g.payload_offset > t.length || g.payload_bytes > t.length - g.payload_offset ||
            g.payload_bytes != ((w - 1) * g.bit_width + 31) / 32 * 4) {
            return Status::malformed_data;
        }
    }
    return Status::success;
}

namespace {

// The ROI clip of one tile: rows [row0, row1) and columns [col0, col1) of the tile, placed at
// output (ox, oy); dst addresses tile column 0 of row row0 in the output. A tile whose rows are
// written whole, have a width the decoder's lane groups cover exactly, and land on 16-byte
// aligned output (and map) rows is marked TSK_FULL: the kernel then stores without checks.
void clip(tsk_decode_task &t, const Roi &roi, std::uint64_t x, std::uint64_t y,
          const tsk_decode_image &im, bool calibrated, std::uint64_t sample) {
    const std::uint64_t rx1 = std::uint64_t{roi.x} + roi.width;
    const std::uint64_t ry1 = std::uint64_t{roi.y} + roi.height;
    t.row0 = static_cast<std::uint16_t>(roi.y > y ? roi.y - y : 0);
    t.row1 = static_cast<std::uint16_t>(ry1 < y + t.height ? ry1 - y : t.height);
    t.col0 = static_cast<std::uint16_t>(roi.x > x ? roi.x - x : 0);
    t.col1 = static_cast<std::uint16_t>(rx1 < x + t.width ? rx1 - x : t.width);
    t.ox = static_cast<std::uint32_t>(x + t.col0 - roi.x);
    t.oy = static_cast<std::uint32_t>(y + t.row0 - roi.y);
    const std::uint64_t esize = calibrated ? 4 : sample;
    // Unsigned wrap-around gives the address before the region when t.ox < t.col0.
    t.dst = im.out + t.oy * im.out_pitch + (std::uint64_t{t.ox} - t.col0) * esize;
    t.pitch = im.out_pitch;
    const bool class_width = t.width == 64 || t.width == 128 || t.width == 256;
    bool aligned = ((t.dst | t.pitch) & 15u) == 0;
    if (calibrated) {
        for (const auto &[map, pitch] : {std::pair{im.offset_map, im.offset_pitch},
                                         std::pair{im.gain_map, im.gain_pitch}}) {
            if (map != 0) {
                aligned = aligned && (((map + t.oy * pitch + std::uint64_t{t.ox} * 4) | pitch) &
                                      15u) == 0;
            }
        }
    }
    if (class_width && t.col0 == 0 && t.col1 == t.width && aligned) {
        t.flags |= TSK_FULL;
    }
}

// Selects the tiles that intersect the region (row-major) and rebases them into the supplied
// bytes (reference plan.cpp:281-349).
Status stage_tiles(const CompressedInput &src, const Roi &roi, std::uint32_t image,
                   std::uint8_t flags, const tsk_decode_image &rec, Draft &d) {
    const ImageMetadata &m = *src.metadata;
    const bool calibrated = (flags & TSK_CALIBRATED) != 0;
    const std::uint64_t sample = m.image.type == PixelType::uint16 ? 2 : 4;
    const std::uint64_t across = tiles_across(m.image, m.tile);
    if (m.tiles.size() != across * tiles_down(m.image, m.tile)) {
        return Status::malformed_data;
    }
    const std::uint64_t left = roi.x / m.tile.width;
    const std::uint64_t right = (std::uint64_t{roi.x} + roi.width - 1) / m.tile.width;
    const std::uint64_t top = roi.y / m.tile.height;
    const std::uint64_t bottom = (std::uint64_t{roi.y} + roi.height - 1) / m.tile.height;
    const std::uint64_t selected = (right - left + 1) * (bottom - top + 1);
    const bool mapped = src.mappings != nullptr || src.mapping_count != 0;
    if (mapped ? src.mappings == nullptr || src.mapping_count != selected
               : m.file_bytes > src.bytes.size) {
        return mapped ? Status::invalid_argument : Status::buffer_too_small;
    }
    std::vector<Range> staged;
    const auto *base = static_cast<const std::uint8_t *>(src.bytes.data);
    std::uint64_t k = 0;
    for (std::uint64_t row = top; row <= bottom; ++row) {
        for (std::uint64_t col = left; col <= right; ++col, ++k) {
            const std::uint64_t index = row * across + col;
            const Status st = check_tile(m, index);
            if (st != Status::success) {
                return st;
            }
            const TileMetadata &t = m.tiles[static_cast<std::size_t>(index)];
            std::uint64_t offset = t.offset;
            if (mapped) {
                const TileMapping &map = src.mappings[k];
                if (map.tile_index != index || map.input_offset % 4 != 0 ||
                    map.input_offset > src.bytes.size ||
                    t.length > src.bytes.size - map.input_offset) {
                    return Status::invalid_argument;
                }
                offset = map.input_offset;
                staged.push_back({static_cast<std::uintptr_t>(offset),
                                  static_cast<std::uintptr_t>(offset + t.length)});
            }
            tsk_decode_task task{};
            task.src = reinterpret_cast<std::uint64_t>(base + offset);
            task.words_or_tile = t.length / 4;
            task.image = image;
            task.width = t.width;
            task.height = t.height;
            task.mode = static_cast<std::uint8_t>(t.mode);
            task.flags = flags | (k == 0 ? TSK_FIRST : 0);
            clip(task, roi, col * m.tile.width, row * m.tile.height, rec, calibrated, sample);
            if (t.mode == TileMode::predict_bitpack) {
                task.rows_at = static_cast<std::uint32_t>(d.rows.size());
                d.rows.resize(d.rows.size() + TSK_ROW_SLOT, 0);
                for (std::uint64_t r = 0; r < t.height; ++r) {
                    const SegmentMetadata &g =
                        m.segments[static_cast<std::size_t>(t.first_segment + r)];
                    // Word index of the row descriptor within the tile payload.
                    d.rows[task.rows_at + r] = static_cast<tsk_row_start>(
                        (g.payload_offset - format::segment_header_bytes) / 4);
                }
            }
            d.tasks.push_back(task);
        }
    }
    std::sort(staged.begin(), staged.end(),
              [](const Range &a, const Range &b) { return a.begin < b.begin; });
    for (std::size_t i = 1; i < staged.size(); ++i) {
        if (staged[i].begin < staged[i - 1].end) {
            return Status::invalid_argument;
        }
    }
    d.tiles_per_image.push_back(selected);
    return Status::success;
}

// Validates and plans one decode item (reference plan.cpp:351-460 per item). With one_type the
// item must have the batch's pixel type (the reference API's rule for one batch); the mixed
// batch API lifts it.
Status draft_decode_item(const BatchItem &item, Operation operation, bool first, bool one_type,
                         Draft &d, bool &mixed) {
    const bool calibrated = operation == Operation::decode_calibrate;
    {
        const CompressedInput &src = item.compressed_input;
        const bool trusted = src.encoder_result != nullptr;
        if (trusted ? src.metadata != nullptr || src.mappings != nullptr || src.mapping_count != 0
                    : src.metadata == nullptr) {
            return Status::invalid_argument;
        }
        const ImageSpec image = trusted ? src.trusted_image : src.metadata->image;
        const TileShape shape = trusted ? src.trusted_tile : src.metadata->tile;
        std::uint64_t bound = 0;
        Status st = compress_bound(image, shape, bound);
        if (st != Status::success) {
            return st;
        }
        if (first) {
            d.type = image.type;
            d.shape = shape;
        }
        if (one_type && image.type != d.type) {
            return Status::invalid_argument;
        }
        d.any_u16 = d.any_u16 || image.type == PixelType::uint16;
        d.any_f32 = d.any_f32 || image.type == PixelType::float32;
        d.any_plain = d.any_plain || !calibrated;
        d.any_calibrated = d.any_calibrated || calibrated;
        mixed = mixed || shape.width != d.shape.width || shape.height != d.shape.height;
        const ImageView &out = item.output;
        st = host::view_ok(out);
        if (st != Status::success) {
            return st;
        }
        Roi roi{0, 0, image.width, image.height};
        if (operation != Operation::decompress) {
            roi = item.roi;
            if (roi.width == 0 || roi.height == 0 ||
                std::uint64_t{roi.x} + roi.width > image.width ||
                std::uint64_t{roi.y} + roi.height > image.height) {
                return Status::invalid_roi;
            }
        }
        if (out.image.type != (calibrated ? PixelType::float32 : image.type) ||
            out.image.width != roi.width || out.image.height != roi.height) {
            return Status::invalid_argument;
        }
        if (calibrated) {
            st = check_calibration(item.calibration, out.image, d);
            if (st != Status::success) {
                return st;
            }
        }
        st = host::byte_range(src.bytes.data, src.bytes.size);
        if (st != Status::success) {
            return st;
        }
        if (src.bytes.data == nullptr || reinterpret_cast<std::uintptr_t>(src.bytes.data) % 4 != 0) {
            return Status::invalid_argument;
        }

        const auto index = static_cast<std::uint32_t>(d.images.size());
        tsk_decode_image rec{};
        rec.out = reinterpret_cast<std::uint64_t>(out.data);
        rec.out_pitch = out.pitch_bytes;
        rec.gain = 1.0f;
        if (calibrated) {
            set_parameters(item.calibration, rec.offset_map, rec.offset_pitch, rec.offset,
                           rec.gain_map, rec.gain_pitch, rec.gain);
        }
        const std::uint64_t out_sample = calibrated ? 4 : (image.type == PixelType::uint16 ? 2 : 4);
        rec.result_bytes = std::uint64_t{roi.width} * roi.height * out_sample;
        rec.archive_width = image.width;
        rec.archive_height = image.height;
        rec.tile_width = shape.width;
        rec.tile_height = shape.height;
        std::uint8_t flags = (image.type == PixelType::float32 ? TSK_F32 : 0) |
                             (calibrated ? TSK_CALIBRATED : 0);
        const std::size_t first_task = d.tasks.size();
        if (trusted) {
            if (reinterpret_cast<std::uintptr_t>(src.encoder_result) % alignof(DeviceResult) != 0) {
                return Status::invalid_argument;
            }
            if (src.bytes.size < bound) {
                return Status::buffer_too_small;
            }
            const std::uint64_t across = tiles_across(image, shape);
            const std::uint64_t top = roi.y / shape.height;
            const std::uint64_t bottom = (std::uint64_t{roi.y} + roi.height - 1) / shape.height;
            const std::uint64_t left = roi.x / shape.width;
            const std::uint64_t right = (std::uint64_t{roi.x} + roi.width - 1) / shape.width;
            for (std::uint64_t row = top; row <= bottom; ++row) {
                for (std::uint64_t col = left; col <= right; ++col) {
                    tsk_decode_task task{};
                    const std::uint64_t x = col * shape.width, y = row * shape.height;
                    task.src = reinterpret_cast<std::uint64_t>(src.bytes.data);
                    task.words_or_tile = row * across + col;
                    task.image = index;
                    task.width = static_cast<std::uint16_t>(
                        std::min<std::uint64_t>(shape.width, image.width - x));
                    task.height = static_cast<std::uint16_t>(
                        std::min<std::uint64_t>(shape.height, image.height - y));
                    task.flags = flags | TSK_TRUSTED;
                    clip(task, roi, x, y, rec, calibrated,
                         image.type == PixelType::uint16 ? 2 : 4);
                    d.tasks.push_back(task);
                }
            }
            d.tiles_per_image.push_back(d.tasks.size() - first_task);
            rec.encoder_result = reinterpret_cast<std::uint64_t>(src.encoder_result);
            rec.capacity = src.bytes.size;
            d.trusted = true;
            d.readable.push_back(range_of(src.encoder_result, sizeof(DeviceResult)));
            d.pointers.push_back(src.encoder_result);
        } else {
            st = stage_tiles(src, roi, index, flags, rec, d);
            if (st != Status::success) {
                return st;
            }
        }
        const std::uint64_t ntasks = d.tasks.size() - first_task;
        if (ntasks > UINT32_MAX) {
            return Status::resource_limit;
        }
        rec.tile_count = static_cast<std::uint32_t>(ntasks);
        d.images.push_back(rec);
        d.readable.push_back(range_of(src.bytes.data, src.bytes.size));
        d.writable.push_back(range_of(out.data, out.capacity_bytes));
        d.pointers.push_back(src.bytes.data);
        d.pointers.push_back(out.data);
    }
    return Status::success;
}

Status draft_decode(const BatchRequest &request, Draft &d) {
    bool mixed = false;
    for (std::uint64_t i = 0; i < request.count; ++i) {
        const Status st = draft_decode_item(request.items[i], request.operation, i == 0, true, d,
                                            mixed);
        if (st != Status::success) {
            return st;
        }
    }
    if (mixed) {
        d.shape = {64, 64}; // the geometry with the most rows bounds every window
    }
    return Status::success;
}

// The reference's window accounting (plan.cpp:467-491, 542-555): maxima of images and tiles over
// sequential windows of at most 4096 tiles.
void window_spec(const std::vector<std::uint64_t> &tiles, WorkspaceSpec &spec) {
    std::uint64_t used = 0, images = 0, count = 0;
    bool open = false;
    auto close = [&]() {
        if (open) {
            spec.image_count = std::max(spec.image_count, images);
            spec.tile_count = std::max(spec.tile_count, count);
        }
    };
    for (std::uint64_t n : tiles) {
        for (std::uint64_t start = 0; start < n;) {
            if (!open || used == kWindowTiles) {
                close();
                open = true;
                used = images = count = 0;
            }
            const std::uint64_t take = std::min<std::uint64_t>(n - start, kWindowTiles - used);
            ++images;
            count += take;
            used += take;
            start += take;
        }
    }
    close();
}

template <typename T>
bool place(std::uint64_t &total, const std::vector<T> &v, std::uint64_t &at) {
    std::uint64_t bytes = 0;
    return host::align_up(total, 256, at) && host::mul(v.size(), sizeof(T), bytes) &&
           host::add(at, bytes, total);
}

template <typename T>
void pack(std::vector<std::uint8_t> &image, std::uint64_t at, const std::vector<T> &v) {
    if (!v.empty()) {
        std::memcpy(image.data() + at, v.data(), v.size() * sizeof(T));
    }
}

// Kernel shape of the plain uint16 decoder (see tsk_decode_config.shape and decode.cu's list).
// The default, shape 15 (four warps in two pairs, each pair staging and decoding its own tiles
// with no producer warp, 16 columns per lane, single-pass rows, two stages per pair, up to six
// CTAs per SM), measured fastest on B200 over all the shapes; TILESTREAM_DECODE_SHAPE overrides
// it for tuning runs.
std::uint32_t decode_shape() {
    static const std::uint32_t shape = [] {
        const char *env = std::getenv("TILESTREAM_DECODE_SHAPE");
        return env != nullptr ? static_cast<std::uint32_t>(std::strtoul(env, nullptr, 10)) %
                                    TSK_DECODE_SHAPES
                              : 15u;
    }();
    return shape;
}

Status finalize(Operation operation, Draft &d, PlanState &plan, cudaStream_t stream);

Status build(const BatchRequest &request, PlanState &plan, cudaStream_t stream) {
    plan.operation = request.operation;
    plan.count = request.count;
    if (request.count == 0) {
        return Status::success;
    }
    Draft d;
    const Status st = request.operation == Operation::compress    ? draft_compress(request, d)
                      : request.operation == Operation::calibrate ? draft_calibrate(request, d)
                                                                  : draft_decode(request, d);
    if (st != Status::success) {
        return st;
    }
    return finalize(request.operation, d, plan, stream);
}

// Everything after the host-side draft: aliasing, device and pointer checks, the reported
// workspace spec, device tables, kernel preload and upload (reference plan.cpp:516-623).
Status finalize(Operation operation, Draft &d, PlanState &plan, cudaStream_t stream) {
    Status st = Status::success;
    plan.type = d.type;
    if (!plan.ranges.assign(std::move(d.writable), std::move(d.readable))) {
        return Status::invalid_argument;
    }
    int pageable = 0;
    if (cudaGetDevice(&plan.device) != cudaSuccess ||
        cudaDeviceGetAttribute(&pageable, cudaDevAttrPageableMemoryAccess, plan.device) !=
            cudaSuccess) {
        return cuda_failure("cudaGetDevice/cudaDeviceGetAttribute");
    }
    plan.pageable = pageable != 0;
    st = stream_device(stream, plan.device);
    if (st != Status::success) {
        return st;
    }
    for (const void *p : d.pointers) {
        st = accessible(p, plan.device, plan.pageable);
        if (st != Status::success) {
            return st;
        }
    }

    plan.spec = {0, 0, d.shape, 0};
    if (operation != Operation::calibrate) {
        window_spec(d.tiles_per_image, plan.spec);
    }
    if (operation == Operation::compress) {
        // This encoder's own device-wide primitive: the look-back flags of every tile.
        plan.spec.scan_temp_bytes = tsk_encode_state_bytes(d.total_tiles);
    }
    st = host::workspace_layout(plan.spec, plan.layout);
    if (st != Status::success) {
        return st;
    }
    if (d.tasks.size() > UINT32_MAX || d.calib_tasks.size() > UINT32_MAX) {
        return Status::resource_limit;
    }

    std::uint64_t total = 0, at_images = 0, at_tasks = 0, at_rows = 0, at_enc = 0, at_cal_images = 0,
                  at_cal_tasks = 0, at_claims = 0;
    const std::vector<std::uint32_t> claims(operation == Operation::compress ||
                                                    operation == Operation::calibrate
                                                ? 0
                                                : 1,
                                            0u); // the decode work queue's counter
    if (!place(total, d.images, at_images) || !place(total, d.tasks, at_tasks) ||
        !place(total, d.rows, at_rows) || !place(total, d.encode_images, at_enc) ||
        !place(total, d.calib_images, at_cal_images) ||
        !place(total, d.calib_tasks, at_cal_tasks) || !place(total, claims, at_claims)) {
        return Status::size_overflow;
    }
    if (cudaMallocAsync(&plan.storage, static_cast<std::size_t>(total), stream) != cudaSuccess) {
        plan.storage = nullptr;
        return cuda_failure("cudaMallocAsync (plan tables)");
    }
    auto *dev = static_cast<std::uint8_t *>(plan.storage);
    plan.images = reinterpret_cast<const tsk_decode_image *>(dev + at_images);
    plan.tasks = reinterpret_cast<const tsk_decode_task *>(dev + at_tasks);
    plan.task_count = static_cast<std::uint32_t>(d.tasks.size());
    plan.rows = reinterpret_cast<const tsk_row_start *>(dev + at_rows);
    plan.trusted = d.trusted;
    plan.encode_images = reinterpret_cast<const tsk_encode_image *>(dev + at_enc);
    plan.total_tiles = d.total_tiles;
    plan.calib_images = reinterpret_cast<const tsk_calib_image *>(dev + at_cal_images);
    plan.calib_tasks = reinterpret_cast<const tsk_calib_task *>(dev + at_cal_tasks);
    plan.calib_task_count = static_cast<std::uint32_t>(d.calib_tasks.size());
    plan.claims = claims.empty() ? nullptr : reinterpret_cast<std::uint32_t *>(dev + at_claims);

    // Load every kernel the plan launches now, so no execution has to (docs/api.md:69).
    int err = 0;
    switch (operation) {
    case Operation::compress:
        err = tsk_encode_prepare(plan.device);
        break;
    case Operation::calibrate:
        err = tsk_calibrate_prepare(plan.device);
        break;
    default:
        // The kernel instance carries only the paths the plan's tiles need.
        plan.config.paths = (d.any_u16 ? TSK_PATH_U16 : 0) | (d.any_f32 ? TSK_PATH_F32 : 0) |
                            (d.any_plain ? TSK_PATH_PLAIN : 0) |
                            (d.any_calibrated ? TSK_PATH_CALIBRATED : 0);
        plan.config.shape = decode_shape();
        err = tsk_decode_prepare(&plan.config, plan.task_count, plan.device);
        break;
    }
    if (err != 0) {
        return cuda_failure("kernel preload", static_cast<cudaError_t>(err));
    }
    // The tables go up in one copy from one host image of the device allocation.
    try {
        std::vector<std::uint8_t> image(static_cast<std::size_t>(total));
        pack(image, at_images, d.images);
        pack(image, at_tasks, d.tasks);
        pack(image, at_rows, d.rows);
        pack(image, at_enc, d.encode_images);
        pack(image, at_cal_images, d.calib_images);
        pack(image, at_cal_tasks, d.calib_tasks);
        pack(image, at_claims, claims);
        if ((total != 0 && cudaMemcpyAsync(plan.storage, image.data(),
                                           static_cast<std::size_t>(total),
                                           cudaMemcpyHostToDevice, stream) != cudaSuccess) ||
            cudaStreamSynchronize(stream) != cudaSuccess) {
            return cuda_failure("plan table upload");
        }
    } catch (const std::bad_alloc &) {
        return Status::resource_limit;
    }
    return Status::success;
}

} // namespace

Status check_execution(const PlanState *plan, Operation operation, MutableBytes workspace,
                       ResultBuffer results, cudaStream_t stream) noexcept {
    if (plan == nullptr || plan->operation != operation) {
        return Status::invalid_argument;
    }
    if (plan->count == 0) {
        return Status::success;
    }
    std::uint64_t result_bytes = 0;
    if (!host::mul(results.count, sizeof(DeviceResult), result_bytes)) {
        return Status::size_overflow;
    }
    Status st = host::byte_range(workspace.data, workspace.size);
    if (st == Status::success) {
        st = host::byte_range(results.data, result_bytes);
    }
    if (st != Status::success) {
        return st;
    }
    if (workspace.size < plan->layout.total || results.count < plan->count) {
        return Status::buffer_too_small;
    }
    if (reinterpret_cast<std::uintptr_t>(workspace.data) % workspace_alignment != 0 ||
        reinterpret_cast<std::uintptr_t>(results.data) % alignof(DeviceResult) != 0) {
        return Status::invalid_argument;
    }
    const Range scratch = range_of(workspace.data, workspace.size);
    const Range records = range_of(results.data, result_bytes);
    if (!plan->ranges.disjoint(scratch) || !plan->ranges.disjoint(records) ||
        host::overlaps(workspace.data, workspace.size, results.data, result_bytes)) {
        return Status::invalid_argument;
    }
    st = stream_device(stream, plan->device);
    if (st == Status::success && workspace.size != 0) {
        st = accessible(workspace.data, plan->device, plan->pageable);
    }
    if (st == Status::success) {
        st = accessible(results.data, plan->device, plan->pageable);
    }
    // A pending error from the caller's own work is left for the caller (docs/api.md:160).
    if (st == Status::success) {
        const cudaError_t pending = cudaPeekAtLastError();
        if (pending != cudaSuccess) {
            log_failure("pending error before enqueue (left for the caller)", pending);
            st = Status::cuda_error;
        }
    }
    return st;
}

} // namespace detail

BatchPlan::BatchPlan(std::unique_ptr<Impl> impl) noexcept : impl_(std::move(impl)) {}
BatchPlan::~BatchPlan() = default;
BatchPlan::BatchPlan(BatchPlan &&) noexcept = default;
BatchPlan &BatchPlan::operator=(BatchPlan &&) noexcept = default;

WorkspaceSpec BatchPlan::workspace_spec() const noexcept {
    return impl_ != nullptr ? impl_->spec : WorkspaceSpec{};
}

namespace detail {

// The host half of prepare_batch for a decode request (drafting and the aliasing rule; no
// device, pointer or allocation step), reported task by task.
Status inspect_decode(const BatchRequest &request, std::vector<TaskSpan> &spans) {
    spans.clear();
    if (request.count > UINT32_MAX) {
        return Status::resource_limit;
    }
    if (request.count != 0 && request.items == nullptr) {
        return Status::invalid_argument;
    }
    if (request.operation != Operation::decompress && request.operation != Operation::decode_roi &&
        request.operation != Operation::decode_calibrate) {
        return Status::invalid_argument;
    }
    if (request.count == 0) {
        return Status::success;
    }
    Draft d;
    Status st = draft_decode(request, d);
    if (st != Status::success) {
        return st;
    }
    RangeSet ranges;
    if (!ranges.assign(d.writable, d.readable)) {
        return Status::invalid_argument;
    }
    spans.reserve(d.tasks.size());
    for (const tsk_decode_task &t : d.tasks) {
        const tsk_decode_image &im = d.images[t.image];
        TaskSpan s;
        s.image = t.image;
        s.mode = t.mode;
        s.flags = t.flags;
        s.width = t.width;
        s.height = t.height;
        if (t.flags & TSK_TRUSTED) {
            s.read_begin = t.src;
            s.read_end = t.src + im.capacity;
        } else {
            s.read_begin = t.src;
            s.read_end = t.src + 4 * t.words_or_tile;
            if (t.mode == TSK_PREDICT) {
                for (std::uint32_t r = 0; r < t.height; ++r) {
                    s.rows_end = std::max<std::uint64_t>(
                        s.rows_end, 4ull * d.rows[t.rows_at + r] + format::segment_header_bytes);
                }
            }
        }
        const std::uint64_t esize = (t.flags & (TSK_F32 | TSK_CALIBRATED)) ? 4 : 2;
        if (t.row1 > t.row0 && t.col1 > t.col0) {
            s.write_begin = t.dst + std::uint64_t{t.col0} * esize;
            s.write_end = t.dst + std::uint64_t(t.row1 - t.row0 - 1) * t.pitch +
                          std::uint64_t{t.col1} * esize;
        }
        spans.push_back(s);
    }
    return Status::success;
}

} // namespace detail

Status prepare_batch(const BatchRequest &request, std::unique_ptr<BatchPlan> &plan,
                     cudaStream_t stream) noexcept {
    if (request.count > UINT32_MAX) {
        return Status::resource_limit;
    }
    if (request.count != 0 && request.items == nullptr) {
        return Status::invalid_argument;
    }
    if (request.operation > Operation::decode_calibrate) {
        return Status::invalid_argument;
    }
    try {
        auto impl = std::make_unique<BatchPlan::Impl>();
        const Status st = detail::build(request, *impl, stream);
        if (st != Status::success) {
            return st;
        }
        plan.reset(new BatchPlan(std::move(impl)));
        return Status::success;
    } catch (const std::bad_alloc &) {
        return Status::resource_limit;
    } catch (const std::length_error &) {
        return Status::resource_limit;
    }
}

namespace {

Status run_decode(const BatchPlan &plan, Operation op, MutableBytes workspace,
                  ResultBuffer results, cudaStream_t stream) noexcept {
    const detail::PlanState *p = PlanAccess::state(plan);
    const Status st = detail::check_execution(p, op, workspace, results, stream);
    if (st != Status::success || p->count == 0) {
        return st;
    }
    auto *records = reinterpret_cast<tsk_result *>(results.data);
    if (p->trusted &&
        cudaMemsetAsync(records, 0, sizeof(tsk_result) * p->count, stream) != cudaSuccess) {
        return detail::cuda_failure("cudaMemsetAsync (results)");
    }
    return detail::cuda_status(
        tsk_decode_launch(p->tasks, p->task_count, p->images, p->rows, records, p->config,
                          p->claims, stream),
        "decode launch");
}

} // namespace

Status decompress_async(const BatchPlan &plan, MutableBytes workspace, ResultBuffer results,
                        cudaStream_t stream) noexcept {
    return run_decode(plan, Operation::decompress, workspace, results, stream);
}

Status decode_roi_async(const BatchPlan &plan, MutableBytes workspace, ResultBuffer results,
                        cudaStream_t stream) noexcept {
    return run_decode(plan, Operation::decode_roi, workspace, results, stream);
}

Status decode_calibrate_async(const BatchPlan &plan, MutableBytes workspace, ResultBuffer results,
                              cudaStream_t stream) noexcept {
    return run_decode(plan, Operation::decode_calibrate, workspace, results, stream);
}

Status compress_async(const BatchPlan &plan, MutableBytes workspace, ResultBuffer results,
                      cudaStream_t stream) noexcept {
    const detail::PlanState *p = PlanAccess::state(plan);
    const Status st = detail::check_execution(p, Operation::compress, workspace, results, stream);
    if (st != Status::success || p->count == 0) {
        return st;
    }
    void *state = static_cast<std::uint8_t *>(workspace.data) + p->layout.temp;
    return detail::cuda_status(tsk_encode_launch(
        p->encode_images, static_cast<std::uint32_t>(p->count), p->total_tiles,
        p->type == PixelType::float32 ? 1u : 0u, state,
        reinterpret_cast<tsk_result *>(results.data), stream), "encode launch");
}

Status calibrate_async(const BatchPlan &plan, MutableBytes workspace, ResultBuffer results,
                       cudaStream_t stream) noexcept {
    const detail::PlanState *p = PlanAccess::state(plan);
    const Status st = detail::check_execution(p, Operation::calibrate, workspace, results, stream);
    if (st != Status::success || p->count == 0) {
        return st;
    }
    return detail::cuda_status(tsk_calibrate_launch(
        p->calib_tasks, p->calib_task_count, p->calib_images, static_cast<std::uint32_t>(p->count),
        reinterpret_cast<tsk_result *>(results.data), stream), "calibrate launch");
}

// ---- mixed batches (include/tilestream/batch.h) ---------------------------------------------

struct MixedBatch::Impl {
    detail::PlanState plan;
    tsk_result *results = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    MixedStats stats;

    ~Impl() {
        if (exec != nullptr) {
            static_cast<void>(cudaGraphExecDestroy(exec));
        }
        if (graph != nullptr) {
            static_cast<void>(cudaGraphDestroy(graph));
        }
    }
};

struct MixedAccess {
    static MixedBatch::Impl *impl(const MixedBatch &b) noexcept {
        return b.impl_.get();
    }
    static std::unique_ptr<MixedBatch> make(std::unique_ptr<MixedBatch::Impl> impl) {
        return std::unique_ptr<MixedBatch>(new MixedBatch(std::move(impl)));
    }
};

MixedBatch::MixedBatch(std::unique_ptr<Impl> impl) noexcept : impl_(std::move(impl)) {}
MixedBatch::~MixedBatch() = default;

namespace {

// One eager execution of a decode plan (used by executions without a graph and by the tuner).
cudaError_t enqueue_decode(const detail::PlanState &p, tsk_result *results, cudaStream_t stream) {
    if (p.trusted) {
        const cudaError_t e =
            cudaMemsetAsync(results, 0, sizeof(tsk_result) * p.count, stream);
        if (e != cudaSuccess) return e;
    }
    return static_cast<cudaError_t>(tsk_decode_launch(p.tasks, p.task_count, p.images, p.rows,
                                                      results, p.config, p.claims, stream));
}

// The tuner's memory: workload key -> (shape, resident CTAs per SM).
struct TuneChoice {
    std::uint32_t shape = 0, per_sm = 0;
};
std::mutex g_tune_mutex;
std::map<std::string, TuneChoice> g_tune_memo;

std::string tune_key(const detail::PlanState &p, int device) {
    cudaDeviceProp prop{};
    static_cast<void>(cudaGetDeviceProperties(&prop, device));
    // The workload signature: device, kernel paths and the task count rounded to a power of two.
    std::uint32_t order = 0;
    while ((1ull << order) < p.task_count) {
        ++order;
    }
    std::string key = prop.name;
    for (char &c : key) {
        if (c == ' ') c = '_';
    }
    // The candidate set is part of the key, so that choices made among other shapes (an older
    // library's cache file) are not replayed.
    return key + "/paths" + std::to_string(p.config.paths) + "/tasks2^" + std::to_string(order) +
           "/shapes" + std::to_string(TSK_DECODE_SHAPES);
}

void load_tune_cache(const char *path) {
    if (path == nullptr) return;
    std::FILE *f = std::fopen(path, "r");
    if (f == nullptr) return;
    char key[512];
    unsigned shape = 0, per_sm = 0;
    while (std::fscanf(f, "%511s %u %u", key, &shape, &per_sm) == 3) {
        g_tune_memo[key] = {shape, per_sm};
    }
    std::fclose(f);
}

void save_tune_cache(const char *path) {
    if (path == nullptr) return;
    std::FILE *f = std::fopen(path, "w");
    if (f == nullptr) return;
    for (const auto &[key, c] : g_tune_memo) {
        std::fprintf(f, "%s %u %u\n", key.c_str(), c.shape, c.per_sm);
    }
    std::fclose(f);
}

// Times candidate configurations (kernel shape x resident CTAs per SM) on the real batch and
// keeps the fastest. Every candidate writes the same outputs and results.
Status autotune(detail::PlanState &p, tsk_result *results, const char *cache, cudaStream_t stream,
                float &best_us) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    load_tune_cache(cache);
    const std::string key = tune_key(p, p.device);
    auto apply = [&](std::uint32_t shape, std::uint32_t per_sm) -> cudaError_t {
        tsk_decode_config c = p.config;
        c.shape = shape;
        int e = tsk_decode_prepare(&c, p.task_count, p.device);
        if (e == 0 && per_sm != 0 && per_sm != c.per_sm) {
            // Fewer (or, up to the occupancy, more) resident CTAs than the shape's default.
            e = tsk_decode_residency(&c, per_sm, p.task_count, p.device);
        }
        if (e != 0) return static_cast<cudaError_t>(e);
        p.config = c;
        return cudaSuccess;
    };
    const auto hit = g_tune_memo.find(key);
    if (hit != g_tune_memo.end()) {
        return detail::cuda_status(apply(hit->second.shape, hit->second.per_sm), "tuned config");
    }
    // The kernel shapes of the batch's instance (kernels/decode.cu, select): nineteen for plain
    // uint16, twelve for plain mixed uint16 + FP32, two for the others.
    const bool plain_u16 = p.config.paths == (TSK_PATH_U16 | TSK_PATH_PLAIN);
    const bool plain_mixed = p.config.paths == (TSK_PATH_U16 | TSK_PATH_F32 | TSK_PATH_PLAIN);
    const std::uint32_t shapes_all[TSK_DECODE_SHAPES] = {0,  1,  2,  3,  4,  5,  6,  7,  8,  9,
                                                         10, 11, 12, 13, 14, 15, 16, 17, 18},
                        shapes_mixed[] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11},
                        shapes_two[] = {0, 2};
    const std::uint32_t *shapes = plain_u16 ? shapes_all : plain_mixed ? shapes_mixed : shapes_two;
    const std::size_t nshapes = plain_u16 ? TSK_DECODE_SHAPES
                                : plain_mixed ? sizeof(shapes_mixed) / sizeof(shapes_mixed[0])
                                              : 2;
    cudaEvent_t start = nullptr, stop = nullptr;
    if (cudaEventCreate(&start) != cudaSuccess || cudaEventCreate(&stop) != cudaSuccess) {
        return detail::cuda_failure("cudaEventCreate");
    }
    TuneChoice best;
    best_us = 0.0f;
    cudaError_t e = cudaSuccess;
    for (std::size_t i = 0; i < nshapes && e == cudaSuccess; ++i) {
        tsk_decode_config probe = p.config;
        probe.shape = shapes[i];
        e = static_cast<cudaError_t>(tsk_decode_prepare(&probe, p.task_count, p.device));
        for (std::uint32_t k = probe.fits; k >= 1 && e == cudaSuccess; --k) {
            e = apply(shapes[i], k);
            if (e == cudaSuccess) e = enqueue_decode(p, results, stream); // warm-up
            constexpr int kRuns = 3;
            if (e == cudaSuccess) e = cudaEventRecord(start, stream);
            for (int r = 0; r < kRuns && e == cudaSuccess; ++r) {
                e = enqueue_decode(p, results, stream);
            }
            if (e == cudaSuccess) e = cudaEventRecord(stop, stream);
            if (e == cudaSuccess) e = cudaEventSynchronize(stop);
            float ms = 0.0f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, start, stop);
            const float us = ms * 1000.0f / kRuns;
            if (e == cudaSuccess && (best_us == 0.0f || us < best_us)) {
                best_us = us;
                best = {shapes[i], k};
            }
            if (k + 2 < probe.fits) {
                break; // fewer CTAs than that never won on this kernel
            }
        }
    }
    cudaEventDestroy(start);
    cudaEventDestroy(stop);
    if (e != cudaSuccess) {
        return detail::cuda_failure("autotune", e);
    }
    g_tune_memo[key] = best;
    save_tune_cache(cache);
    return detail::cuda_status(apply(best.shape, best.per_sm), "tuned config");
}

} // namespace

Status prepare_mixed_batch(const MixedItem *items, std::uint64_t count, ResultBuffer results,
                           const MixedOptions &options, std::unique_ptr<MixedBatch> &batch,
                           cudaStream_t stream) noexcept {
    if (count > UINT32_MAX) {
        return Status::resource_limit;
    }
    if (count != 0 && items == nullptr) {
        return Status::invalid_argument;
    }
    try {
        auto impl = std::make_unique<MixedBatch::Impl>();
        detail::PlanState &plan = impl->plan;
        plan.operation = Operation::decode_roi;
        plan.count = count;
        if (count != 0) {
            detail::Draft d;
            bool mixed = false;
            for (std::uint64_t i = 0; i < count; ++i) {
                const Operation op = items[i].operation;
                if (op != Operation::decompress && op != Operation::decode_roi &&
                    op != Operation::decode_calibrate) {
                    return Status::invalid_argument;
                }
                const Status st = detail::draft_decode_item(items[i].item, op, i == 0, false, d,
                                                            mixed);
                if (st != Status::success) {
                    return st;
                }
            }
            if (mixed) {
                d.shape = {64, 64};
            }
            std::uint64_t result_bytes = 0;
            if (!host::mul(results.count, sizeof(DeviceResult), result_bytes)) {
                return Status::size_overflow;
            }
            Status st = host::byte_range(results.data, result_bytes);
            if (st != Status::success) {
                return st;
            }
            if (results.count < count) {
                return Status::buffer_too_small;
            }
            if (reinterpret_cast<std::uintptr_t>(results.data) % alignof(DeviceResult) != 0) {
                return Status::invalid_argument;
            }
            d.writable.push_back(detail::range_of(results.data, result_bytes));
            d.pointers.push_back(results.data);
            st = detail::finalize(Operation::decode_roi, d, plan, stream);
            if (st != Status::success) {
                return st;
            }
            impl->results = reinterpret_cast<tsk_result *>(results.data);
            if (options.shape >= static_cast<std::int32_t>(TSK_DECODE_SHAPES)) {
                return Status::invalid_argument;
            }
            if (options.shape >= 0) {
                plan.config.shape = static_cast<std::uint32_t>(options.shape);
                const int e = tsk_decode_prepare(&plan.config, plan.task_count, plan.device);
                if (e != 0) {
                    return detail::cuda_failure("kernel shape", static_cast<cudaError_t>(e));
                }
            } else if (options.autotune) {
                const char *cache = options.tune_cache != nullptr
                                        ? options.tune_cache
                                        : std::getenv("TILESTREAM_TUNE_CACHE");
                st = autotune(plan, impl->results, cache, stream, impl->stats.tuned_us);
                if (st != Status::success) {
                    return st;
                }
            }
            if (options.graph) {
                const int e = tsk_decode_graph(plan.tasks, plan.task_count, plan.images, plan.rows,
                                               impl->results, static_cast<std::uint32_t>(count),
                                               plan.trusted ? 1 : 0, plan.config, plan.claims,
                                               &impl->graph, &impl->exec);
                if (e != 0) {
                    impl->graph = nullptr;
                    impl->exec = nullptr;
                    return detail::cuda_failure("graph instantiation",
                                                static_cast<cudaError_t>(e));
                }
                // Upload the graph now so that the first execution does no set-up work.
                if (cudaGraphUpload(impl->exec, stream) != cudaSuccess ||
                    cudaStreamSynchronize(stream) != cudaSuccess) {
                    return detail::cuda_failure("cudaGraphUpload");
                }
            }
            impl->stats = {plan.task_count, plan.config.shape, plan.config.grid,
                           plan.config.per_sm, impl->exec != nullptr ? 1u : 0u,
                           impl->stats.tuned_us};
        }
        batch = MixedAccess::make(std::move(impl));
        return Status::success;
    } catch (const std::bad_alloc &) {
        return Status::resource_limit;
    } catch (const std::length_error &) {
        return Status::resource_limit;
    }
}

Status run_mixed_batch(const MixedBatch &batch, cudaStream_t stream) noexcept {
    const MixedBatch::Impl *impl = MixedAccess::impl(batch);
    if (impl == nullptr) {
        return Status::invalid_argument;
    }
    const detail::PlanState &p = impl->plan;
    if (p.count == 0) {
        return Status::success;
    }
    Status st = detail::stream_device(stream, p.device);
    if (st == Status::success && cudaPeekAtLastError() != cudaSuccess) {
        st = Status::cuda_error; // left for the caller
    }
    if (st != Status::success) {
        return st;
    }
    if (impl->exec != nullptr) {
        return detail::cuda_status(cudaGraphLaunch(impl->exec, stream), "cudaGraphLaunch");
    }
    return detail::cuda_status(enqueue_decode(p, impl->results, stream), "decode launch");
}

std::uint32_t decode_shape_count() noexcept {
    return TSK_DECODE_SHAPES;
}

MixedStats mixed_batch_stats(const MixedBatch &batch) noexcept {
    const MixedBatch::Impl *impl = MixedAccess::impl(batch);
    return impl != nullptr ? impl->stats : MixedStats{};
}

} // namespace tilestream::cuda
