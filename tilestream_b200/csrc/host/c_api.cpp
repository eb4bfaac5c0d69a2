// The C entry layer of include/tilestream_c.h over the C++ API.
#include <tilestream/batch.h>
#include <tilestream/cpu.h>
#include <tilestream/cuda.h>
#include <tilestream/info.h>
#include <tilestream/serve.h>
#include <tilestream/staging.h>
#include <tilestream/tiff.h>
#include <tilestream/unparsed.h>
#include <tilestream_c.h>

#include "plan.h"

#include <cstddef>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <type_traits>
#include <vector>

namespace ts = tilestream;

// Each C record has the layout of the C++ record it mirrors.
#define TS_SAME_LAYOUT(C, CPP)                                                                    \
    static_assert(sizeof(C) == sizeof(CPP) && alignof(C) == alignof(CPP), #C " layout")
TS_SAME_LAYOUT(ts_image_spec, ts::ImageSpec);
TS_SAME_LAYOUT(ts_tile_shape, ts::TileShape);
TS_SAME_LAYOUT(ts_roi, ts::Roi);
TS_SAME_LAYOUT(ts_const_bytes, ts::ConstBytes);
TS_SAME_LAYOUT(ts_mutable_bytes, ts::MutableBytes);
TS_SAME_LAYOUT(ts_const_image_view, ts::ConstImageView);
TS_SAME_LAYOUT(ts_image_view, ts::ImageView);
TS_SAME_LAYOUT(ts_device_result, ts::DeviceResult);
TS_SAME_LAYOUT(ts_parameter, ts::cuda::Parameter);
TS_SAME_LAYOUT(ts_calibration, ts::cuda::Calibration);
TS_SAME_LAYOUT(ts_tile_mapping, ts::cuda::TileMapping);
TS_SAME_LAYOUT(ts_roi_staging, ts::cuda::RoiStaging);
TS_SAME_LAYOUT(ts_parse_limits, ts::ParseLimits);
TS_SAME_LAYOUT(ts_tiff_read_limits, ts::io::TiffReadLimits);
TS_SAME_LAYOUT(ts_unparsed_file, ts::cuda::UnparsedFile);
static_assert(offsetof(ts_unparsed_file, output) == offsetof(ts::cuda::UnparsedFile, output));
TS_SAME_LAYOUT(ts_workspace_spec, ts::WorkspaceSpec);
TS_SAME_LAYOUT(ts_tile_metadata, ts::TileMetadata);
TS_SAME_LAYOUT(ts_segment_metadata, ts::SegmentMetadata);
TS_SAME_LAYOUT(ts_compressed_input, ts::cuda::CompressedInput);
TS_SAME_LAYOUT(ts_batch_item, ts::cuda::BatchItem);
TS_SAME_LAYOUT(ts_batch_request, ts::cuda::BatchRequest);
TS_SAME_LAYOUT(ts_result_buffer, ts::cuda::ResultBuffer);
static_assert(offsetof(ts_batch_item, compressed_input) ==
              offsetof(ts::cuda::BatchItem, compressed_input));
static_assert(offsetof(ts_batch_item, calibration) == offsetof(ts::cuda::BatchItem, calibration));
static_assert(offsetof(ts_compressed_input, metadata) ==
              offsetof(ts::cuda::CompressedInput, metadata));
static_assert(offsetof(ts_compressed_input, trusted_tile) ==
              offsetof(ts::cuda::CompressedInput, trusted_tile));
static_assert(sizeof(ts::cuda::DeviceTile) == 40 && sizeof(ts::cuda::DeviceSegment) == 16 &&
              sizeof(ts::DeviceResult) == 16);
static_assert(std::is_trivially_copyable_v<ts::cuda::DeviceImage> &&
              std::is_standard_layout_v<ts::cuda::DeviceBatch>);

TS_SAME_LAYOUT(ts_mixed_item, ts::cuda::MixedItem);
TS_SAME_LAYOUT(ts_task_span, ts::cuda::detail::TaskSpan);
TS_SAME_LAYOUT(ts_mixed_stats, ts::cuda::MixedStats);
static_assert(offsetof(ts_mixed_item, item) == offsetof(ts::cuda::MixedItem, item));

TS_SAME_LAYOUT(ts_serve_request, ts::cuda::ServeRequest);
TS_SAME_LAYOUT(ts_serve_options, ts::cuda::ServeOptions);
TS_SAME_LAYOUT(ts_serve_stats, ts::cuda::ServeStats);
TS_SAME_LAYOUT(ts_serve_outcome, ts::cuda::ServeOutcome);
static_assert(offsetof(ts_serve_request, arrival_us) ==
              offsetof(ts::cuda::ServeRequest, arrival_us));
static_assert(offsetof(ts_serve_options, serial) == offsetof(ts::cuda::ServeOptions, serial));
static_assert(offsetof(ts_serve_stats, output_bytes) ==
              offsetof(ts::cuda::ServeStats, output_bytes));
static_assert(offsetof(ts_serve_outcome, result) == offsetof(ts::cuda::ServeOutcome, result));
static_assert(std::is_trivially_copyable_v<ts::cuda::ServeRequest> &&
              std::is_trivially_copyable_v<ts::cuda::ServeOutcome>);

struct ts_metadata {
    ts::ImageMetadata value;
};

struct ts_mixed_batch {
    std::unique_ptr<ts::cuda::MixedBatch> batch;
};

struct ts_plan {
    std::unique_ptr<ts::cuda::BatchPlan> plan;
};

struct ts_tiff_image {
    ts::io::TiffImage value;
};

struct ts_server {
    std::unique_ptr<ts::cuda::Server> server;
};

namespace {

template <typename To, typename From> To as(const From &from) {
    static_assert(sizeof(To) == sizeof(From));
    To to;
    std::memcpy(static_cast<void *>(&to), &from, sizeof(To));
    return to;
}

int code(ts::Status s) {
    return static_cast<int>(s);
}

cudaStream_t stream_of(void *s) {
    return static_cast<cudaStream_t>(s);
}

ts::ParseLimits limits_of(const ts_parse_limits *l) {
    return l != nullptr ? as<ts::ParseLimits>(*l) : ts::ParseLimits{};
}

} // namespace

extern "C" {

int ts_image_span(ts_image_spec image, uint64_t pitch_bytes, uint64_t *bytes) {
    return code(ts::image_span(as<ts::ImageSpec>(image), pitch_bytes, *bytes));
}

int ts_compress_bound(ts_image_spec image, ts_tile_shape tile, uint64_t *bytes) {
    return code(ts::compress_bound(as<ts::ImageSpec>(image), as<ts::TileShape>(tile), *bytes));
}

int ts_workspace_size(const ts_workspace_spec *spec, uint64_t *bytes) {
    return code(ts::workspace_size(as<ts::WorkspaceSpec>(*spec), *bytes));
}

int ts_parse_metadata(ts_const_bytes source, const ts_parse_limits *limits, ts_metadata **out) {
    std::unique_ptr<ts_metadata> m(new (std::nothrow) ts_metadata);
    if (!m) {
        return code(ts::Status::resource_limit);
    }
    const ts::Status st =
        ts::parse_metadata(as<ts::ConstBytes>(source), limits_of(limits), m->value);
    if (st == ts::Status::success) {
        *out = m.release();
    }
    return code(st);
}

int ts_metadata_create(ts_image_spec image, ts_tile_shape tile, uint64_t file_bytes,
                       const ts_tile_metadata *tiles, uint64_t tile_count,
                       const ts_segment_metadata *segments, uint64_t segment_count,
                       ts_metadata **out) {
    if ((tiles == nullptr && tile_count != 0) || (segments == nullptr && segment_count != 0)) {
        return code(ts::Status::invalid_argument);
    }
    try {
        auto m = std::make_unique<ts_metadata>();
        m->value.image = as<ts::ImageSpec>(image);
        m->value.tile = as<ts::TileShape>(tile);
        m->value.file_bytes = file_bytes;
        m->value.tiles.resize(tile_count);
        m->value.segments.resize(segment_count);
        if (tile_count != 0) {
            std::memcpy(static_cast<void *>(m->value.tiles.data()), tiles,
                        tile_count * sizeof(ts_tile_metadata));
        }
        if (segment_count != 0) {
            std::memcpy(static_cast<void *>(m->value.segments.data()), segments,
                        segment_count * sizeof(ts_segment_metadata));
        }
        *out = m.release();
        return code(ts::Status::success);
    } catch (...) {
        return code(ts::Status::resource_limit);
    }
}

void ts_metadata_destroy(ts_metadata *metadata) {
    delete metadata;
}

void ts_metadata_info(const ts_metadata *m, ts_image_spec *image, ts_tile_shape *tile,
                      uint64_t *file_bytes, uint64_t *tile_count, uint64_t *segment_count) {
    if (image) *image = as<ts_image_spec>(m->value.image);
    if (tile) *tile = as<ts_tile_shape>(m->value.tile);
    if (file_bytes) *file_bytes = m->value.file_bytes;
    if (tile_count) *tile_count = m->value.tiles.size();
    if (segment_count) *segment_count = m->value.segments.size();
}

const ts_tile_metadata *ts_metadata_tiles(const ts_metadata *m) {
    return reinterpret_cast<const ts_tile_metadata *>(m->value.tiles.data());
}

const ts_segment_metadata *ts_metadata_segments(const ts_metadata *m) {
    return reinterpret_cast<const ts_segment_metadata *>(m->value.segments.data());
}

int ts_cpu_compress(ts_const_image_view input, ts_tile_shape tile, ts_mutable_bytes output,
                    uint64_t *bytes_written) {
    return code(ts::cpu::compress(as<ts::ConstImageView>(input), as<ts::TileShape>(tile),
                                  as<ts::MutableBytes>(output), *bytes_written));
}

int ts_cpu_decompress(ts_const_bytes input, ts_image_view output, const ts_parse_limits *limits) {
    return code(ts::cpu::decompress(as<ts::ConstBytes>(input), as<ts::ImageView>(output),
                                    limits_of(limits)));
}

int ts_prepare_batch(const ts_batch_request *request, ts_plan **plan, void *stream) {
    if (request == nullptr || plan == nullptr) {
        return code(ts::Status::invalid_argument);
    }
    try {
        ts::cuda::BatchRequest r = as<ts::cuda::BatchRequest>(*request);
        std::vector<ts::cuda::BatchItem> items;
        if (request->items != nullptr && request->count <= UINT32_MAX) {
            items.resize(request->count);
            for (uint64_t i = 0; i < request->count; ++i) {
                items[i] = as<ts::cuda::BatchItem>(request->items[i]);
                const ts_metadata *m = request->items[i].compressed_input.metadata;
                items[i].compressed_input.metadata = m != nullptr ? &m->value : nullptr;
            }
            r.items = items.data();
        }
        auto holder = std::make_unique<ts_plan>();
        const ts::Status st = ts::cuda::prepare_batch(r, holder->plan, stream_of(stream));
        if (st == ts::Status::success) {
            delete *plan;
            *plan = holder.release();
        }
        return code(st);
    } catch (...) {
        return code(ts::Status::resource_limit);
    }
}

int ts_inspect_decode(const ts_batch_request *request, ts_task_span *spans, uint64_t capacity,
                      uint64_t *count) {
    if (request == nullptr || count == nullptr || (capacity != 0 && spans == nullptr)) {
        return code(ts::Status::invalid_argument);
    }
    try {
        ts::cuda::BatchRequest r = as<ts::cuda::BatchRequest>(*request);
        std::vector<ts::cuda::BatchItem> items;
        if (request->items != nullptr && request->count <= UINT32_MAX) {
            items.resize(request->count);
            for (uint64_t i = 0; i < request->count; ++i) {
                items[i] = as<ts::cuda::BatchItem>(request->items[i]);
                const ts_metadata *m = request->items[i].compressed_input.metadata;
                items[i].compressed_input.metadata = m != nullptr ? &m->value : nullptr;
            }
            r.items = items.data();
        }
        std::vector<ts::cuda::detail::TaskSpan> found;
        const ts::Status st = ts::cuda::detail::inspect_decode(r, found);
        *count = found.size();
        for (uint64_t i = 0; i < found.size() && i < capacity; ++i) {
            spans[i] = as<ts_task_span>(found[i]);
        }
        return code(st);
    } catch (...) {
        return code(ts::Status::resource_limit);
    }
}

void ts_plan_destroy(ts_plan *plan) {
    delete plan;
}

int ts_plan_workspace_spec(const ts_plan *plan, ts_workspace_spec *spec) {
    if (plan == nullptr || !plan->plan || spec == nullptr) {
        return code(ts::Status::invalid_argument);
    }
    *spec = as<ts_workspace_spec>(plan->plan->workspace_spec());
    return 0;
}

#define TS_EXECUTOR(name)                                                                         \
    int ts_##name(const ts_plan *plan, ts_mutable_bytes workspace, ts_result_buffer results,      \
                  void *stream) {                                                                 \
        if (plan == nullptr || !plan->plan) {                                                     \
            return code(ts::Status::invalid_argument);                                            \
        }                                                                                         \
        return code(ts::cuda::name(*plan->plan, as<ts::MutableBytes>(workspace),                  \
                                   as<ts::cuda::ResultBuffer>(results), stream_of(stream)));      \
    }
TS_EXECUTOR(compress_async)
TS_EXECUTOR(decompress_async)
TS_EXECUTOR(decode_roi_async)
TS_EXECUTOR(calibrate_async)
TS_EXECUTOR(decode_calibrate_async)
#undef TS_EXECUTOR

// Same contract as DeviceBuffer::allocate (cuda.h:124-125); the caller owns the memory and frees
// it with ts_device_release.
int ts_device_allocate(uint64_t bytes, void *stream, void **data) {
    if (bytes > ts::max_bytes) {
        return code(ts::Status::size_overflow);
    }
    if (bytes == 0) {
        *data = nullptr;
        return 0;
    }
    void *p = nullptr;
    if (cudaMallocAsync(&p, static_cast<std::size_t>(bytes), stream_of(stream)) != cudaSuccess) {
        return code(ts::cuda::detail::cuda_failure());
    }
    if (reinterpret_cast<std::uintptr_t>(p) % ts::workspace_alignment != 0) {
        static_cast<void>(cudaFreeAsync(p, stream_of(stream)));
        return code(ts::Status::cuda_error);
    }
    *data = p;
    return 0;
}

int ts_device_release(void *data, void *stream) {
    if (data == nullptr) {
        return 0;
    }
    return code(ts::cuda::detail::cuda_status(cudaFreeAsync(data, stream_of(stream))));
}

int ts_synchronize(void *stream) {
    return code(ts::cuda::synchronize(stream_of(stream)));
}

const char *ts_version(void) {
    return ts::version();
}

int ts_info_json(char *buf, uint64_t capacity, uint64_t *needed) {
    try {
        const std::string s = ts::info_json();
        if (needed != nullptr) {
            *needed = s.size() + 1;
        }
        if (buf != nullptr && capacity >= s.size() + 1) {
            std::memcpy(buf, s.c_str(), s.size() + 1);
            return 0;
        }
        return code(ts::Status::buffer_too_small);
    } catch (...) {
        return code(ts::Status::resource_limit);
    }
}

} // extern "C"

extern "C" int ts_prepare_mixed_batch(const ts_mixed_item *items, uint64_t count,
                                      ts_result_buffer results, const ts_mixed_options *options,
                                      ts_mixed_batch **batch, void *stream) {
    if (batch == nullptr || (count != 0 && items == nullptr)) {
        return code(ts::Status::invalid_argument);
    }
    if (count > UINT32_MAX) {
        return code(ts::Status::resource_limit);
    }
    try {
        std::vector<ts::cuda::MixedItem> converted(count);
        for (uint64_t i = 0; i < count; ++i) {
            converted[i] = as<ts::cuda::MixedItem>(items[i]);
            const ts_metadata *m = items[i].item.compressed_input.metadata;
            converted[i].item.compressed_input.metadata = m != nullptr ? &m->value : nullptr;
        }
        ts::cuda::MixedOptions o;
        if (options != nullptr) {
            o.graph = options->graph != 0;
            o.autotune = options->autotune != 0;
            o.tune_cache = options->tune_cache;
            o.shape = options->shape;
        }
        auto holder = std::make_unique<ts_mixed_batch>();
        const ts::Status st = ts::cuda::prepare_mixed_batch(
            converted.data(), count, as<ts::cuda::ResultBuffer>(results), o, holder->batch,
            stream_of(stream));
        if (st == ts::Status::success) {
            delete *batch;
            *batch = holder.release();
        }
        return code(st);
    } catch (...) {
        return code(ts::Status::resource_limit);
    }
}

extern "C" uint32_t ts_decode_shape_count(void) {
    return ts::cuda::decode_shape_count();
}

extern "C" int ts_run_mixed_batch(const ts_mixed_batch *batch, void *stream) {
    if (batch == nullptr || !batch->batch) {
        return code(ts::Status::invalid_argument);
    }
    return code(ts::cuda::run_mixed_batch(*batch->batch, stream_of(stream)));
}

extern "C" int ts_mixed_batch_stats(const ts_mixed_batch *batch, ts_mixed_stats *stats) {
    if (batch == nullptr || !batch->batch || stats == nullptr) {
        return code(ts::Status::invalid_argument);
    }
    *stats = as<ts_mixed_stats>(ts::cuda::mixed_batch_stats(*batch->batch));
    return 0;
}

extern "C" void ts_mixed_batch_destroy(ts_mixed_batch *batch) {
    delete batch;
}

extern "C" int ts_server_create(const ts_serve_options *options, ts_server **server) {
    if (server == nullptr) {
        return code(ts::Status::invalid_argument);
    }
    try {
        const ts::cuda::ServeOptions o =
            options != nullptr ? as<ts::cuda::ServeOptions>(*options) : ts::cuda::ServeOptions{};
        auto holder = std::make_unique<ts_server>();
        const ts::Status st = ts::cuda::Server::create(o, holder->server);
        if (st == ts::Status::success) {
            delete *server;
            *server = holder.release();
        }
        return code(st);
    } catch (...) {
        return code(ts::Status::resource_limit);
    }
}

extern "C" int ts_server_add_archive(ts_server *server, ts_const_bytes device_bytes,
                                     const ts_metadata *metadata, uint32_t *id) {
    if (server == nullptr || !server->server || metadata == nullptr || id == nullptr) {
        return code(ts::Status::invalid_argument);
    }
    return code(server->server->add_archive(as<ts::ConstBytes>(device_bytes), metadata->value,
                                            *id));
}

extern "C" int ts_server_seal(ts_server *server) {
    if (server == nullptr || !server->server) {
        return code(ts::Status::invalid_argument);
    }
    return code(server->server->seal());
}

extern "C" int ts_server_run(ts_server *server, const ts_serve_request *requests, uint64_t count,
                             ts_serve_outcome *outcomes, ts_serve_stats *stats) {
    if (server == nullptr || !server->server || stats == nullptr) {
        return code(ts::Status::invalid_argument);
    }
    ts::cuda::ServeStats s;
    const ts::Status st = server->server->run(
        reinterpret_cast<const ts::cuda::ServeRequest *>(requests), count,
        reinterpret_cast<ts::cuda::ServeOutcome *>(outcomes), s);
    *stats = as<ts_serve_stats>(s);
    return code(st);
}

extern "C" int ts_server_pool(const ts_server *server, ts_mutable_bytes *pool) {
    if (server == nullptr || !server->server || pool == nullptr) {
        return code(ts::Status::invalid_argument);
    }
    *pool = as<ts_mutable_bytes>(server->server->pool());
    return 0;
}

extern "C" int ts_server_start(ts_server *server, uint32_t max_outstanding) {
    if (server == nullptr || !server->server) {
        return code(ts::Status::invalid_argument);
    }
    return code(server->server->start(max_outstanding));
}

extern "C" int ts_server_submit(ts_server *server, const ts_serve_request *request,
                                uint64_t *ticket) {
    if (server == nullptr || !server->server || request == nullptr || ticket == nullptr) {
        return code(ts::Status::invalid_argument);
    }
    return code(server->server->submit(*reinterpret_cast<const ts::cuda::ServeRequest *>(request),
                                       *ticket));
}

extern "C" int ts_server_wait(ts_server *server, uint64_t ticket, uint64_t timeout_us,
                              ts_serve_outcome *outcome, int *done) {
    if (server == nullptr || !server->server || outcome == nullptr || done == nullptr) {
        return code(ts::Status::invalid_argument);
    }
    bool finished = false;
    const ts::Status st = server->server->wait(
        ticket, timeout_us, *reinterpret_cast<ts::cuda::ServeOutcome *>(outcome), finished);
    *done = finished ? 1 : 0;
    return code(st);
}

extern "C" int ts_server_release(ts_server *server, uint64_t ticket) {
    if (server == nullptr || !server->server) {
        return code(ts::Status::invalid_argument);
    }
    return code(server->server->release(ticket));
}

extern "C" int ts_server_stop(ts_server *server) {
    if (server == nullptr || !server->server) {
        return code(ts::Status::invalid_argument);
    }
    return code(server->server->stop());
}

extern "C" void ts_server_destroy(ts_server *server) {
    delete server;
}

extern "C" int ts_roi_staging_size(const ts_metadata *metadata, ts_roi roi, ts_roi_staging *out) {
    if (metadata == nullptr || out == nullptr) {
        return code(ts::Status::invalid_argument);
    }
    ts::cuda::RoiStaging r;
    const ts::Status st = ts::cuda::roi_staging_size(metadata->value, as<ts::Roi>(roi), r);
    if (st == ts::Status::success) {
        *out = as<ts_roi_staging>(r);
    }
    return code(st);
}

extern "C" int ts_stage_roi_tiles(const ts_metadata *metadata, ts_roi roi, ts_const_bytes archive,
                                  ts_mutable_bytes staging, ts_tile_mapping *mappings,
                                  uint64_t mapping_capacity, void *stream, ts_roi_staging *out) {
    if (metadata == nullptr || out == nullptr) {
        return code(ts::Status::invalid_argument);
    }
    ts::cuda::RoiStaging r;
    const ts::Status st = ts::cuda::stage_roi_tiles(
        metadata->value, as<ts::Roi>(roi), as<ts::ConstBytes>(archive),
        as<ts::MutableBytes>(staging), reinterpret_cast<ts::cuda::TileMapping *>(mappings),
        mapping_capacity, stream_of(stream), r);
    if (st == ts::Status::success) {
        *out = as<ts_roi_staging>(r);
    }
    return code(st);
}

// Allocation-free one-image encode (declared in include/tilestream_c.h; no counterpart in the
// reference). Host checks follow compress_async's (draft_compress and check_execution in
// plan.cpp), then the image is encoded with the static scratch of encode.cu.
extern "C" uint64_t ts_compress_noalloc_max_tiles(void) {
    return tsk_encode_static_max_tiles();
}

extern "C" int ts_compress_noalloc(ts_const_image_view input_c, ts_tile_shape tile_c,
                                   ts_mutable_bytes output_c, ts_device_result *result,
                                   void *stream_v) {
    namespace d = ts::cuda::detail;
    const auto input = as<ts::ConstImageView>(input_c);
    const auto tile = as<ts::TileShape>(tile_c);
    const auto output = as<ts::MutableBytes>(output_c);
    const cudaStream_t stream = stream_of(stream_v);
    ts::Status st = ts::host::view_ok(input);
    if (st != ts::Status::success) {
        return code(st);
    }
    std::uint64_t bound = 0;
    st = ts::compress_bound(input.image, tile, bound);
    if (st != ts::Status::success) {
        return code(st);
    }
    st = ts::host::byte_range(output.data, output.size);
    if (st != ts::Status::success) {
        return code(st);
    }
    if (output.data == nullptr || reinterpret_cast<std::uintptr_t>(output.data) % 4 != 0) {
        return code(ts::Status::invalid_argument);
    }
    if (output.size < bound) {
        return code(ts::Status::buffer_too_small);
    }
    if (result == nullptr || reinterpret_cast<std::uintptr_t>(result) % alignof(ts::DeviceResult)) {
        return code(ts::Status::invalid_argument);
    }
    if (ts::host::overlaps(input.data, input.capacity_bytes, output.data, output.size) ||
        ts::host::overlaps(result, sizeof(ts::DeviceResult), output.data, output.size) ||
        ts::host::overlaps(result, sizeof(ts::DeviceResult), input.data, input.capacity_bytes)) {
        return code(ts::Status::invalid_argument);
    }
    tsk_encode_image image{};
    image.columns = ts::host::ceil_div(input.image.width, tile.width);
    image.tile_count = image.columns * ts::host::ceil_div(input.image.height, tile.height);
    if (image.tile_count > tsk_encode_static_max_tiles()) {
        return code(ts::Status::resource_limit);
    }
    int device = 0, pageable = 0;
    if (cudaGetDevice(&device) != cudaSuccess ||
        cudaDeviceGetAttribute(&pageable, cudaDevAttrPageableMemoryAccess, device) != cudaSuccess) {
        return code(d::cuda_failure("cudaGetDevice/cudaDeviceGetAttribute"));
    }
    st = d::stream_device(stream, device);
    for (const void *p : {input.data, static_cast<const void *>(output.data),
                          static_cast<const void *>(result)}) {
        if (st == ts::Status::success) {
            st = d::accessible(p, device, pageable != 0);
        }
    }
    if (st == ts::Status::success && cudaPeekAtLastError() != cudaSuccess) {
        st = ts::Status::cuda_error; // the caller's pending error is left for the caller
    }
    if (st != ts::Status::success) {
        return code(st);
    }
    image.input = reinterpret_cast<std::uint64_t>(input.data);
    image.pitch = input.pitch_bytes;
    image.output = reinterpret_cast<std::uint64_t>(output.data);
    image.first_tile = 0;
    image.width = input.image.width;
    image.height = input.image.height;
    image.tile_width = tile.width;
    image.tile_height = tile.height;
    image.type = static_cast<std::uint32_t>(input.image.type);
    return code(d::cuda_status(
        tsk_encode_static_launch(&image, reinterpret_cast<tsk_result *>(result), stream),
        "allocation-free encode launch"));
}

extern "C" int ts_read_tiff(const char *path, const ts_tiff_read_limits *limits,
                            ts_tiff_image **image) {
    if (image == nullptr) {
        return code(ts::Status::invalid_argument);
    }
    try {
        auto holder = std::make_unique<ts_tiff_image>();
        const ts::io::TiffReadLimits l =
            limits != nullptr ? as<ts::io::TiffReadLimits>(*limits) : ts::io::TiffReadLimits{};
        const ts::Status st = ts::io::read_tiff(path, holder->value, l);
        if (st == ts::Status::success) {
            delete *image;
            *image = holder.release();
        }
        return code(st);
    } catch (...) {
        return code(ts::Status::resource_limit);
    }
}

extern "C" int ts_tiff_image_pixels(const ts_tiff_image *image, ts_image_spec *spec,
                                    uint64_t *pitch_bytes, const void **pixels, uint64_t *bytes) {
    if (image == nullptr || spec == nullptr || pitch_bytes == nullptr || pixels == nullptr ||
        bytes == nullptr) {
        return code(ts::Status::invalid_argument);
    }
    *spec = as<ts_image_spec>(image->value.image);
    *pitch_bytes = image->value.pitch_bytes;
    *pixels = image->value.pixels.data();
    *bytes = image->value.pixels.size();
    return 0;
}

extern "C" void ts_tiff_image_destroy(ts_tiff_image *image) {
    delete image;
}

extern "C" int ts_write_tiff(const char *path, ts_const_image_view image,
                             const ts_tiff_write_options *options) {
    ts::io::TiffWriteOptions o;
    if (options != nullptr) {
        if (options->compression > 1) {
            return code(ts::Status::invalid_argument);
        }
        o.bigtiff = options->bigtiff != 0;
        o.compression = static_cast<ts::io::TiffCompression>(options->compression);
        o.horizontal_predictor = options->horizontal_predictor != 0;
        o.tile_width = options->tile_width;
        o.tile_height = options->tile_height;
        o.deflate_level = options->deflate_level;
    }
    return code(ts::io::write_tiff(path, as<ts::ConstImageView>(image), o));
}

extern "C" int ts_decode_unparsed_async(const ts_unparsed_file *files, uint64_t count,
                                        ts_result_buffer results, void *stream) {
    return code(ts::cuda::decode_unparsed_async(
        reinterpret_cast<const ts::cuda::UnparsedFile *>(files), count,
        as<ts::cuda::ResultBuffer>(results), static_cast<cudaStream_t>(stream)));
}
