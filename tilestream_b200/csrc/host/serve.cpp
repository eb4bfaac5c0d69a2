// The ROI serving loop of include/tilestream/serve.h.
//
// Resident state (built once): per archive a table of tile templates, which are decode tasks
// with the archive-dependent fields set, and for predictive tiles a row-start slot. Both sit in
// one device allocation with the archive table. A request costs the host one 64-byte record in
// the launch's parameter block. The kernel turns (request, tile l of its ROI) into a task with
// the same clip that the planner applies per tile (reference plan.cpp:281-349 selects the
// intersecting tiles, tests/cuda_decoder_test.cpp:19-31).
//
// run() drives the loop on the calling thread over a known request stream; start() drives the
// same loop on a thread of its own over requests that callers submit while it runs. On each
// pass the loop:
//   1. polls the in-flight launches' events and records the completion time of their requests;
//   2. frees the output memory of finished requests (unless outputs are retained);
//   3. admits the requests that have arrived, in arrival order, while the output pool has room;
//   4. launches them as one batch (at most max_batch requests) on a free stream.
// Output memory is a ring over the pool: allocations are made in admission order and freed in
// any order, and the ring's tail advances over freed blocks.
#include <tilestream/serve.h>

#include "../kernels/tasks.h"
#include "plan.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

namespace tilestream::cuda {
namespace {

using Clock = std::chrono::steady_clock;

double micros(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::micro>(b - a).count();
}

constexpr std::uint32_t kMaxInflight = 16;

// Output memory in admission order; blocks are freed in any order.
class Ring {
  public:
    explicit Ring(std::uint64_t capacity) : cap_(capacity) {}

    // Reserves size bytes (a multiple of 256); returns the block's sequence number.
    bool alloc(std::uint64_t size, std::uint64_t &offset, std::uint64_t &seq) {
        if (size > cap_) {
            return false;
        }
        if (live_.empty()) {
            head_ = 0;
            offset = 0;
        } else {
            const std::uint64_t tail = live_.front().offset;
            const bool wrapped = live_.back().offset < tail;
            if (!wrapped) {
                // Free: [head, cap) and [0, tail).
                if (cap_ - head_ >= size) {
                    offset = head_;
                } else if (tail >= size) {
                    offset = 0;
                } else {
                    return false;
                }
            } else {
                // Free: [head, tail).
                if (tail - head_ >= size) {
                    offset = head_;
                } else {
                    return false;
                }
            }
        }
        head_ = offset + size;
        seq = first_ + live_.size();
        live_.push_back({offset, false});
        return true;
    }

    void release(std::uint64_t seq) {
        live_[static_cast<std::size_t>(seq - first_)].freed = true;
        while (!live_.empty() && live_.front().freed) {
            live_.pop_front();
            ++first_;
        }
    }

  private:
    struct Block {
        std::uint64_t offset;
        bool freed;
    };
    std::uint64_t cap_;
    std::uint64_t head_ = 0;
    std::uint64_t first_ = 0; // sequence number of live_.front()
    std::deque<Block> live_;
};

struct ArchiveEntry {
    ConstBytes bytes;
    const ImageMetadata *metadata = nullptr;
    std::uint64_t first_tile = 0; // index of tile 0 in the template table
    std::uint64_t across = 0, down = 0;
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    bool busy = false;
    std::uint64_t r0 = 0, r1 = 0; // requests [r0, r1)
};

// One request of a session, from submit() to release().
struct Ticket {
    ServeRequest request;
    std::uint64_t bytes = 0, tiles = 0;
    std::uint64_t seq = 0;  // its block in the ring, when placed
    bool placed = false;    // output memory allocated
    bool done = false;      // outcome final
    Clock::time_point submitted;
    ServeOutcome outcome;
};

// The state shared by the session thread and the callers, guarded by `mu`.
struct Session {
    std::mutex mu;
    std::condition_variable completed; // callers waiting for a request
    std::condition_variable wake;      // the session thread, idle
    std::thread worker;
    std::unordered_map<std::uint64_t, Ticket> tickets;
    std::deque<std::uint64_t> queue; // submitted, not yet admitted, in submission order
    std::vector<std::vector<std::uint64_t>> launched; // per slot: its batch's tickets
    std::unique_ptr<Ring> ring;
    std::uint64_t next_ticket = 1;
    std::uint32_t max_outstanding = 0;
    bool running = false, stopping = false;
    Status failure = Status::success;
    tsk_result *device_records = nullptr; // per slot: max_batch records
    tsk_result *host_records = nullptr;   // pinned copies of them
};

// The launch record of request q, output at `out` with rows `pitch` bytes apart.
void fill_record(tsk_serve_request &rec, const ServeRequest &q, const ArchiveEntry &a,
                 std::uint64_t out, std::uint64_t pitch) {
    const TileShape tile = a.metadata->tile;
    rec.out = out;
    rec.out_pitch = pitch;
    rec.archive = q.archive;
    rec.x = q.roi.x;
    rec.y = q.roi.y;
    rec.width = q.roi.width;
    rec.height = q.roi.height;
    rec.left = q.roi.x / tile.width;
    rec.top = q.roi.y / tile.height;
    rec.across = static_cast<std::uint32_t>(
        (std::uint64_t{q.roi.x} + q.roi.width - 1) / tile.width - rec.left + 1);
    rec.flags = q.calibrated != 0 ? TSK_CALIBRATED : 0;
    rec.offset = q.offset;
    rec.gain = q.gain;
}

} // namespace

struct Server::Impl {
    ServeOptions options;
    int device = 0;
    std::uint8_t *pool = nullptr;
    std::vector<ArchiveEntry> archives;
    std::vector<tsk_decode_task> templates; // host copies until seal()
    std::vector<tsk_row_start> rows;
    bool all_u16 = true;
    bool sealed = false;
    void *tables = nullptr; // device: archive table, templates, row starts
    const tsk_serve_archive *dev_archives = nullptr;
    const tsk_row_start *dev_rows = nullptr;
    std::uint32_t grid = 0;
    std::vector<Slot> slots;
    Session session;

    ~Impl() {
        end_session();
        if (session.device_records != nullptr) cudaFree(session.device_records);
        if (session.host_records != nullptr) cudaFreeHost(session.host_records);
        for (Slot &s : slots) {
            if (s.done != nullptr) cudaEventDestroy(s.done);
            if (s.stream != nullptr) cudaStreamDestroy(s.stream);
        }
        if (tables != nullptr) cudaFree(tables);
        if (pool != nullptr) cudaFree(pool);
    }

    Status run_batched(const ServeRequest *requests, std::uint64_t count, ServeOutcome *outcomes,
                       ServeStats &stats);
    Status run_serial(const ServeRequest *requests, std::uint64_t count, ServeOutcome *outcomes,
                      ServeStats &stats);
    void session_loop();
    void settle_queued(Status status);
    void end_session() {
        {
            std::lock_guard<std::mutex> lock(session.mu);
            session.stopping = true;
        }
        session.wake.notify_all();
        if (session.worker.joinable()) session.worker.join();
    }
};

Server::Server(std::unique_ptr<Impl> impl) noexcept : impl_(std::move(impl)) {}
Server::~Server() = default;

MutableBytes Server::pool() const noexcept {
    return {impl_->pool, impl_->options.output_pool_bytes};
}

Status Server::create(const ServeOptions &options, std::unique_ptr<Server> &out) noexcept {
    if (options.output_pool_bytes == 0 || options.max_batch == 0 ||
        options.max_batch > TSK_SERVE_MAX_BATCH || options.max_inflight == 0 ||
        options.max_inflight > kMaxInflight || options.max_batch_tiles == 0 ||
        options.max_batch_tiles > UINT32_MAX) {
        return Status::invalid_argument;
    }
    std::unique_ptr<Impl> impl(new (std::nothrow) Impl);
    if (impl == nullptr) {
        return Status::resource_limit;
    }
    impl->options = options;
    if (cudaGetDevice(&impl->device) != cudaSuccess) {
        return detail::cuda_failure("cudaGetDevice");
    }
    if (cudaMalloc(reinterpret_cast<void **>(&impl->pool),
                   static_cast<std::size_t>(options.output_pool_bytes)) != cudaSuccess) {
        impl->pool = nullptr;
        cudaGetLastError();
        return Status::resource_limit;
    }
    impl->slots.resize(options.max_inflight);
    for (Slot &s : impl->slots) {
        if (cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming) != cudaSuccess) {
            return detail::cuda_failure("serving streams");
        }
    }
    out.reset(new (std::nothrow) Server(std::move(impl)));
    return out != nullptr ? Status::success : Status::resource_limit;
}

Status Server::add_archive(ConstBytes device_bytes, const ImageMetadata &m,
                           std::uint32_t &id) noexcept {
    Impl &s = *impl_;
    if (s.sealed) {
        return Status::invalid_argument;
    }
    if (device_bytes.data == nullptr || m.file_bytes > device_bytes.size ||
        !host::supported_tile(m.tile) || m.image.width == 0 || m.image.height == 0) {
        return Status::invalid_argument;
    }
    if (m.image.type != PixelType::uint16 && m.image.type != PixelType::float32) {
        return Status::unsupported_type;
    }
    const Status acc = detail::accessible(device_bytes.data, s.device, false);
    if (acc != Status::success) {
        return acc;
    }
    ArchiveEntry a;
    a.bytes = device_bytes;
    a.metadata = &m;
    a.across = host::ceil_div(m.image.width, m.tile.width);
    a.down = host::ceil_div(m.image.height, m.tile.height);
    if (m.tiles.size() != a.across * a.down) {
        return Status::malformed_data;
    }
    a.first_tile = s.templates.size();
    const bool f32 = m.image.type == PixelType::float32;
    const auto *base = static_cast<const std::uint8_t *>(device_bytes.data);
    try {
        s.templates.reserve(s.templates.size() + m.tiles.size());
        for (std::uint64_t i = 0; i < m.tiles.size(); ++i) {
            const Status st = detail::check_tile(m, i);
            if (st != Status::success) {
                s.templates.resize(static_cast<std::size_t>(a.first_tile));
                return st;
            }
            const TileMetadata &t = m.tiles[static_cast<std::size_t>(i)];
            tsk_decode_task task{};
            task.src = reinterpret_cast<std::uint64_t>(base + t.offset);
            task.words_or_tile = t.length / 4;
            task.width = t.width;
            task.height = t.height;
            task.mode = static_cast<std::uint8_t>(t.mode);
            task.flags = f32 ? TSK_F32 : 0;
            if (t.mode == TileMode::predict_bitpack) {
                if (s.rows.size() + TSK_ROW_SLOT > UINT32_MAX) {
                    s.templates.resize(static_cast<std::size_t>(a.first_tile));
                    return Status::resource_limit;
                }
                task.rows_at = static_cast<std::uint32_t>(s.rows.size());
                s.rows.resize(s.rows.size() + TSK_ROW_SLOT, 0);
                for (std::uint64_t r = 0; r < t.height; ++r) {
                    const SegmentMetadata &g =
                        m.segments[static_cast<std::size_t>(t.first_segment + r)];
                    s.rows[task.rows_at + r] = static_cast<tsk_row_start>(
                        (g.payload_offset - format::segment_header_bytes) / 4);
                }
            }
            s.templates.push_back(task);
        }
        s.archives.push_back(a);
    } catch (const std::bad_alloc &) {
        return Status::resource_limit;
    }
    s.all_u16 = s.all_u16 && !f32;
    id = static_cast<std::uint32_t>(s.archives.size() - 1);
    return Status::success;
}

Status Server::seal() noexcept {
    Impl &s = *impl_;
    if (s.sealed || s.archives.empty()) {
        return Status::invalid_argument;
    }
    const std::uint64_t n = s.archives.size();
    const std::uint64_t at_tpl = (n * sizeof(tsk_serve_archive) + 255) / 256 * 256;
    const std::uint64_t at_rows =
        at_tpl + (s.templates.size() * sizeof(tsk_decode_task) + 255) / 256 * 256;
    const std::uint64_t total = at_rows + s.rows.size() * sizeof(tsk_row_start) + 16;
    if (cudaMalloc(&s.tables, static_cast<std::size_t>(total)) != cudaSuccess) {
        s.tables = nullptr;
        cudaGetLastError();
        return Status::resource_limit;
    }
    auto *dev = static_cast<std::uint8_t *>(s.tables);
    std::vector<tsk_serve_archive> table(static_cast<std::size_t>(n));
    for (std::size_t i = 0; i < table.size(); ++i) {
        const ArchiveEntry &a = s.archives[i];
        table[i].tiles = reinterpret_cast<std::uint64_t>(dev + at_tpl) +
                         a.first_tile * sizeof(tsk_decode_task);
        table[i].tiles_across = static_cast<std::uint32_t>(a.across);
        table[i].tile_width = a.metadata->tile.width;
        table[i].tile_height = a.metadata->tile.height;
        table[i].type = static_cast<std::uint32_t>(a.metadata->image.type);
    }
    if (cudaMemcpy(dev, table.data(), table.size() * sizeof(tsk_serve_archive),
                   cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dev + at_tpl, s.templates.data(),
                   s.templates.size() * sizeof(tsk_decode_task),
                   cudaMemcpyHostToDevice) != cudaSuccess ||
        (!s.rows.empty() && cudaMemcpy(dev + at_rows, s.rows.data(),
                                       s.rows.size() * sizeof(tsk_row_start),
                                       cudaMemcpyHostToDevice) != cudaSuccess)) {
        return detail::cuda_failure("serving table upload");
    }
    s.dev_archives = reinterpret_cast<const tsk_serve_archive *>(dev);
    s.dev_rows = reinterpret_cast<const tsk_row_start *>(dev + at_rows);
    const int e = tsk_serve_prepare(s.all_u16 ? 1 : 0, s.device, &s.grid);
    if (e != 0) {
        return detail::cuda_failure("serving kernel preload", static_cast<cudaError_t>(e));
    }
    // The templates live on the device now; the host copies are not needed again.
    std::vector<tsk_decode_task>().swap(s.templates);
    std::vector<tsk_row_start>().swap(s.rows);
    s.sealed = true;
    return Status::success;
}

namespace {

// Host checks of one request; fills the output geometry.
Status check_request(const ServeRequest &q, const std::vector<ArchiveEntry> &archives,
                     std::uint64_t pool_bytes, std::uint64_t &pitch, std::uint64_t &bytes,
                     std::uint64_t &tiles) {
    if (q.archive >= archives.size()) {
        return Status::invalid_argument;
    }
    const ImageMetadata &m = *archives[q.archive].metadata;
    const Roi &r = q.roi;
    if (r.width == 0 || r.height == 0 || r.x >= m.image.width || r.y >= m.image.height ||
        r.width > m.image.width - r.x || r.height > m.image.height - r.y) {
        return Status::invalid_roi;
    }
    const std::uint64_t esize = (q.calibrated != 0 || m.image.type == PixelType::float32) ? 4 : 2;
    pitch = (std::uint64_t{r.width} * esize + 15) / 16 * 16;
    bytes = (pitch * r.height + 255) / 256 * 256;
    if (bytes > pool_bytes) {
        return Status::buffer_too_small;
    }
    const std::uint64_t across = (std::uint64_t{r.x} + r.width - 1) / m.tile.width -
                                 r.x / m.tile.width + 1;
    const std::uint64_t down = (std::uint64_t{r.y} + r.height - 1) / m.tile.height -
                               r.y / m.tile.height + 1;
    tiles = across * down;
    // Task indexes of a launch are 32-bit.
    return tiles < (1ull << 31) ? Status::success : Status::resource_limit;
}

// Nearest-rank percentile of sorted values.
double rank(const std::vector<double> &v, double p) {
    if (v.empty()) return 0.0;
    std::size_t k = static_cast<std::size_t>(p / 100.0 * static_cast<double>(v.size()) + 0.999999);
    k = std::min(std::max<std::size_t>(k, 1), v.size());
    return v[k - 1];
}

void summarize(std::uint64_t count, const ServeOutcome *outcomes, double wall_us,
               ServeStats &stats) {
    std::vector<double> lat;
    lat.reserve(static_cast<std::size_t>(count));
    double sum = 0;
    for (std::uint64_t i = 0; i < count; ++i) {
        if (outcomes[i].batch_size != 0) {
            lat.push_back(outcomes[i].latency_us);
            sum += outcomes[i].latency_us;
            if (outcomes[i].result.status == Status::success) {
                stats.output_bytes += outcomes[i].result.bytes_written;
            }
        }
    }
    std::sort(lat.begin(), lat.end());
    stats.completed = lat.size();
    stats.wall_us = wall_us;
    stats.p50_us = rank(lat, 50);
    stats.p90_us = rank(lat, 90);
    stats.p99_us = rank(lat, 99);
    stats.max_us = lat.empty() ? 0.0 : lat.back();
    stats.mean_us = lat.empty() ? 0.0 : sum / static_cast<double>(lat.size());
    stats.throughput_rps = wall_us > 0 ? static_cast<double>(lat.size()) / wall_us * 1e6 : 0.0;
    stats.decoded_gbs = wall_us > 0 ? static_cast<double>(stats.output_bytes) / wall_us / 1e3 : 0.0;
}

} // namespace

Status Server::run(const ServeRequest *requests, std::uint64_t count, ServeOutcome *outcomes,
                   ServeStats &stats) noexcept {
    Impl &s = *impl_;
    if (!s.sealed || (count != 0 && (requests == nullptr || outcomes == nullptr))) {
        return Status::invalid_argument;
    }
    {
        std::lock_guard<std::mutex> lock(s.session.mu);
        if (s.session.running) {
            return Status::invalid_argument;
        }
    }
    for (std::uint64_t i = 1; i < count; ++i) {
        if (!(requests[i].arrival_us >= requests[i - 1].arrival_us)) {
            return Status::invalid_argument;
        }
    }
    stats = ServeStats{};
    for (std::uint64_t i = 0; i < count; ++i) {
        outcomes[i] = ServeOutcome{};
    }
    try {
        return s.options.serial != 0 ? s.run_serial(requests, count, outcomes, stats)
                                     : s.run_batched(requests, count, outcomes, stats);
    } catch (const std::bad_alloc &) {
        return Status::resource_limit;
    }
}

Status Server::Impl::run_batched(const ServeRequest *requests, std::uint64_t count,
                                 ServeOutcome *outcomes, ServeStats &stats) {
    // Host-side geometry of every request; refused ones are settled before the clock starts.
    std::vector<std::uint64_t> bytes(static_cast<std::size_t>(count)),
        tiles(static_cast<std::size_t>(count)), seq(static_cast<std::size_t>(count));
    for (std::uint64_t i = 0; i < count; ++i) {
        const Status st = check_request(requests[i], archives, options.output_pool_bytes,
                                        outcomes[i].output_pitch, bytes[i], tiles[i]);
        if (st != Status::success) {
            outcomes[i].result.status = st;
            ++stats.rejected;
            bytes[i] = tiles[i] = 0;
        }
    }
    tsk_result *results = nullptr;
    if (count != 0 && cudaMalloc(reinterpret_cast<void **>(&results),
                                 count * sizeof(tsk_result)) != cudaSuccess) {
        cudaGetLastError();
        return Status::resource_limit;
    }
    struct Free {
        tsk_result *p;
        ~Free() {
            if (p != nullptr) cudaFree(p);
        }
    } free_results{results};
    // Cleared on a serving stream (the launches' streams do not wait for the legacy one).
    if (count != 0 &&
        (cudaMemsetAsync(results, 0xff, count * sizeof(tsk_result), slots[0].stream) !=
             cudaSuccess ||
         cudaStreamSynchronize(slots[0].stream) != cudaSuccess)) {
        return detail::cuda_failure("cudaMemsetAsync (serving results)");
    }

    Ring ring(options.output_pool_bytes);
    std::vector<char> stalled(static_cast<std::size_t>(count), 0);
    std::vector<Clock::time_point> launched(static_cast<std::size_t>(count));
    tsk_serve_batch batch;
    const std::uint32_t limit = options.max_batch;
    std::uint64_t next = 0, done = 0, inflight = 0;
    Status failure = Status::success;
    const Clock::time_point t0 = Clock::now();
    Clock::time_point last = t0;
    auto arrival = [&](std::uint64_t i) {
        return t0 + std::chrono::duration_cast<Clock::duration>(
                        std::chrono::duration<double, std::micro>(requests[i].arrival_us));
    };
    while (done < count && failure == Status::success) {
        // 1-2. Completions.
        for (Slot &slot : slots) {
            if (!slot.busy) continue;
            const cudaError_t q = cudaEventQuery(slot.done);
            if (q == cudaErrorNotReady) continue;
            if (q != cudaSuccess) {
                failure = detail::cuda_failure("serving batch", q);
                break;
            }
            const Clock::time_point now = Clock::now();
            last = now;
            for (std::uint64_t r = slot.r0; r < slot.r1; ++r) {
                if (outcomes[r].batch_size == 0) continue; // refused on the host
                outcomes[r].latency_us = micros(arrival(r), now);
                if (options.retain_outputs == 0) ring.release(seq[r]);
            }
            done += slot.r1 - slot.r0;
            slot.busy = false;
            --inflight;
        }
        if (failure != Status::success) break;
        // Refused requests at the head complete immediately.
        while (next < count && bytes[next] == 0 && arrival(next) <= Clock::now()) {
            ++next;
            ++done;
        }
        // 3-4. Admission and launch.
        Slot *free_slot = nullptr;
        for (Slot &slot : slots) {
            if (!slot.busy) {
                free_slot = &slot;
                break;
            }
        }
        if (free_slot == nullptr || next >= count) continue;
        const Clock::time_point now = Clock::now();
        const std::uint64_t r0 = next;
        std::uint32_t n = 0;
        std::uint64_t ntasks = 0;
        while (next < count && n < limit && arrival(next) <= now) {
            std::uint64_t offset = 0;
            if (bytes[next] != 0) {
                if (ntasks + tiles[next] > options.max_batch_tiles && n != 0) break;
                if (!ring.alloc(bytes[next], offset, seq[next])) {
                    if (options.retain_outputs != 0) {
                        // Retained outputs are never freed during the run: this one cannot fit.
                        outcomes[next].result.status = Status::resource_limit;
                        ++stats.rejected;
                        bytes[next] = 0;
                    } else {
                        if (!stalled[next]) {
                            stalled[next] = 1;
                            ++stats.stalls;
                        }
                        break;
                    }
                }
            }
            if (bytes[next] != 0) {
                const ServeRequest &q = requests[next];
                tsk_serve_request &rec = batch.requests[n];
                fill_record(rec, q, archives[q.archive],
                            reinterpret_cast<std::uint64_t>(pool) + offset,
                            outcomes[next].output_pitch);
                ntasks += tiles[next];
                rec.task_end = static_cast<std::uint32_t>(ntasks);
                outcomes[next].output_offset = offset;
            } else {
                // A refused request inside the batch's range: no tasks, no output.
                tsk_serve_request &rec = batch.requests[n];
                std::memset(&rec, 0, sizeof(rec));
                rec.task_end = static_cast<std::uint32_t>(ntasks);
            }
            ++n;
            ++next;
        }
        if (n == 0) continue;
        // Refused requests at the tail are settled outside the batch.
        while (n != 0 && bytes[next - 1] == 0) {
            --n;
            --next;
        }
        if (n == 0) continue;
        batch.count = n;
        batch.ntasks = static_cast<std::uint32_t>(ntasks);
        const int e = tsk_serve_launch(&batch, dev_archives, dev_rows, results + r0, grid,
                                       all_u16 ? 1 : 0, free_slot->stream);
        if (e != 0 || cudaEventRecord(free_slot->done, free_slot->stream) != cudaSuccess) {
            failure = detail::cuda_failure("serving launch", static_cast<cudaError_t>(e));
            break;
        }
        const Clock::time_point at = Clock::now();
        for (std::uint64_t r = r0; r < next; ++r) {
            if (bytes[r] == 0) continue;
            outcomes[r].queued_us = micros(arrival(r), at);
            outcomes[r].batch_size = n;
        }
        free_slot->busy = true;
        free_slot->r0 = r0;
        free_slot->r1 = next;
        ++inflight;
        stats.max_inflight = std::max<std::uint64_t>(stats.max_inflight, inflight);
        ++stats.batches;
        stats.tiles += ntasks;
    }
    // Drain whatever is still running (after a failure).
    for (Slot &slot : slots) {
        if (slot.busy) {
            cudaEventSynchronize(slot.done);
            slot.busy = false;
        }
    }
    if (failure != Status::success) {
        return failure;
    }
    std::vector<tsk_result> host(static_cast<std::size_t>(count));
    if (count != 0 && cudaMemcpy(host.data(), results, count * sizeof(tsk_result),
                                 cudaMemcpyDeviceToHost) != cudaSuccess) {
        return detail::cuda_failure("cudaMemcpy (serving results)");
    }
    for (std::uint64_t i = 0; i < count; ++i) {
        if (outcomes[i].batch_size != 0) {
            outcomes[i].result.status = static_cast<Status>(host[i].status);
            outcomes[i].result.bytes_written = host[i].bytes_written;
        }
    }
    std::uint64_t served = 0;
    for (std::uint64_t i = 0; i < count; ++i) {
        served += outcomes[i].batch_size != 0 ? 1 : 0;
    }
    stats.mean_batch = stats.batches != 0 ? static_cast<double>(served) / stats.batches : 0.0;
    summarize(count, outcomes, micros(t0, last), stats);
    return Status::success;
}

Status Server::Impl::run_serial(const ServeRequest *requests, std::uint64_t count,
                                ServeOutcome *outcomes, ServeStats &stats) {
    std::vector<std::uint64_t> bytes(static_cast<std::size_t>(count)),
        tiles(static_cast<std::size_t>(count));
    for (std::uint64_t i = 0; i < count; ++i) {
        const Status st = check_request(requests[i], archives, options.output_pool_bytes,
                                        outcomes[i].output_pitch, bytes[i], tiles[i]);
        if (st != Status::success) {
            outcomes[i].result.status = st;
            ++stats.rejected;
            bytes[i] = 0;
        }
    }
    cudaStream_t stream = slots[0].stream;
    DeviceResult *results = nullptr;
    if (count != 0 && cudaMalloc(reinterpret_cast<void **>(&results),
                                 count * sizeof(DeviceResult)) != cudaSuccess) {
        cudaGetLastError();
        return Status::resource_limit;
    }
    struct Free {
        void *p;
        ~Free() {
            if (p != nullptr) cudaFree(p);
        }
    } free_results{results}, free_workspace{nullptr};
    // One workspace for every plan: the largest per tile shape and kind of request, found by
    // planning the largest request of each before the clock starts.
    std::uint64_t workspace_bytes = 0;
    auto item_of = [&](std::uint64_t i, std::uint64_t offset) {
        const ServeRequest &q = requests[i];
        const ArchiveEntry &a = archives[q.archive];
        BatchItem item;
        item.compressed_input.bytes = a.bytes;
        item.compressed_input.metadata = a.metadata;
        const PixelType type = q.calibrated != 0 ? PixelType::float32 : a.metadata->image.type;
        item.output.data = pool + offset;
        item.output.image = {type, q.roi.width, q.roi.height};
        item.output.pitch_bytes = outcomes[i].output_pitch;
        item.output.capacity_bytes = bytes[i];
        item.roi = q.roi;
        item.calibration.offset.scalar = q.offset;
        item.calibration.gain.scalar = q.gain;
        return item;
    };
    auto operation_of = [&](std::uint64_t i) {
        return requests[i].calibrated != 0 ? Operation::decode_calibrate : Operation::decode_roi;
    };
    {
        std::vector<std::uint64_t> largest;
        for (std::uint64_t i = 0; i < count; ++i) {
            if (bytes[i] == 0) continue;
            bool seen = false;
            for (std::uint64_t &j : largest) {
                const TileShape a = archives[requests[i].archive].metadata->tile;
                const TileShape b = archives[requests[j].archive].metadata->tile;
                if (a.width == b.width && a.height == b.height &&
                    operation_of(i) == operation_of(j)) {
                    seen = true;
                    if (tiles[i] > tiles[j]) j = i;
                }
            }
            if (!seen) largest.push_back(i);
        }
        for (std::uint64_t i : largest) {
            const BatchItem item = item_of(i, 0);
            const BatchRequest req{operation_of(i), &item, 1, {}};
            std::unique_ptr<BatchPlan> plan;
            Status st = prepare_batch(req, plan, stream);
            std::uint64_t need = 0;
            if (st == Status::success) st = workspace_size(plan->workspace_spec(), need);
            if (st != Status::success) return st;
            workspace_bytes = std::max(workspace_bytes, need);
        }
    }
    if (workspace_bytes != 0 &&
        cudaMalloc(&free_workspace.p, static_cast<std::size_t>(workspace_bytes)) != cudaSuccess) {
        cudaGetLastError();
        return Status::resource_limit;
    }
    const MutableBytes workspace{free_workspace.p, workspace_bytes};
    Ring ring(options.output_pool_bytes);
    const Clock::time_point t0 = Clock::now();
    Clock::time_point last = t0;
    for (std::uint64_t i = 0; i < count; ++i) {
        if (bytes[i] == 0) continue;
        const Clock::time_point arrival =
            t0 + std::chrono::duration_cast<Clock::duration>(
                     std::chrono::duration<double, std::micro>(requests[i].arrival_us));
        while (Clock::now() < arrival) {
        }
        std::uint64_t offset = 0, block = 0;
        if (!ring.alloc(bytes[i], offset, block)) {
            ++stats.rejected; // retained outputs filled the pool
            outcomes[i].result.status = Status::resource_limit;
            continue;
        }
        const BatchItem item = item_of(i, offset);
        const Operation op = operation_of(i);
        const BatchRequest req{op, &item, 1, {}};
        std::unique_ptr<BatchPlan> plan;
        Status st = prepare_batch(req, plan, stream);
        if (st == Status::success) {
            outcomes[i].queued_us = micros(arrival, Clock::now());
            const ResultBuffer rb{results + i, 1};
            st = op == Operation::decode_calibrate
                     ? decode_calibrate_async(*plan, workspace, rb, stream)
                     : decode_roi_async(*plan, workspace, rb, stream);
        }
        if (st == Status::success) st = synchronize(stream);
        if (st != Status::success) return st;
        last = Clock::now();
        outcomes[i].latency_us = micros(arrival, last);
        outcomes[i].output_offset = offset;
        outcomes[i].batch_size = 1;
        ++stats.batches;
        stats.tiles += tiles[i];
        plan.reset();
        if (options.retain_outputs == 0) ring.release(block);
    }
    std::vector<DeviceResult> host(static_cast<std::size_t>(count));
    if (count != 0 && cudaMemcpy(host.data(), results, count * sizeof(DeviceResult),
                                 cudaMemcpyDeviceToHost) != cudaSuccess) {
        return detail::cuda_failure("cudaMemcpy (serving results)");
    }
    for (std::uint64_t i = 0; i < count; ++i) {
        if (outcomes[i].batch_size != 0) outcomes[i].result = host[i];
    }
    stats.max_inflight = stats.batches != 0 ? 1 : 0;
    stats.mean_batch = stats.batches != 0 ? 1.0 : 0.0;
    summarize(count, outcomes, micros(t0, last), stats);
    return Status::success;
}

// ---- sessions ---------------------------------------------------------------------------

Status Server::start(std::uint32_t max_outstanding) noexcept {
    Impl &s = *impl_;
    Session &S = s.session;
    std::lock_guard<std::mutex> lock(S.mu);
    if (!s.sealed || S.running || s.options.serial != 0 || max_outstanding == 0) {
        return Status::invalid_argument;
    }
    if (S.worker.joinable()) {
        S.worker.join(); // a loop that ended on a failure
    }
    const std::uint64_t records = std::uint64_t{s.options.max_inflight} * s.options.max_batch;
    if (S.device_records == nullptr) {
        if (cudaMalloc(reinterpret_cast<void **>(&S.device_records),
                       records * sizeof(tsk_result)) != cudaSuccess) {
            S.device_records = nullptr;
            cudaGetLastError();
            return Status::resource_limit;
        }
        if (cudaMallocHost(reinterpret_cast<void **>(&S.host_records),
                           records * sizeof(tsk_result)) != cudaSuccess) {
            S.host_records = nullptr;
            cudaGetLastError();
            return Status::resource_limit;
        }
    }
    try {
        S.ring = std::make_unique<Ring>(s.options.output_pool_bytes);
        S.tickets.clear();
        S.queue.clear();
        S.launched.assign(s.slots.size(), {});
        for (std::vector<std::uint64_t> &ids : S.launched) {
            ids.reserve(s.options.max_batch); // no allocation on the session thread
        }
        S.max_outstanding = max_outstanding;
        S.failure = Status::success;
        S.stopping = false;
        S.running = true;
        S.worker = std::thread([&s] { s.session_loop(); });
    } catch (...) {
        S.running = false;
        return Status::resource_limit;
    }
    return Status::success;
}

Status Server::submit(const ServeRequest &request, std::uint64_t &ticket) noexcept {
    Impl &s = *impl_;
    Session &S = s.session;
    Ticket t;
    t.request = request;
    const Status st = check_request(request, s.archives, s.options.output_pool_bytes,
                                    t.outcome.output_pitch, t.bytes, t.tiles);
    if (st != Status::success) {
        return st;
    }
    {
        std::lock_guard<std::mutex> lock(S.mu);
        if (!S.running || S.stopping) {
            return Status::invalid_argument;
        }
        if (S.failure != Status::success) {
            return S.failure;
        }
        if (S.tickets.size() >= S.max_outstanding) {
            return Status::resource_limit;
        }
        t.submitted = Clock::now();
        try {
            const std::uint64_t id = S.next_ticket;
            S.tickets.emplace(id, t);
            S.queue.push_back(id);
            ++S.next_ticket;
            ticket = id;
        } catch (const std::bad_alloc &) {
            S.tickets.erase(S.next_ticket);
            return Status::resource_limit;
        }
    }
    S.wake.notify_one();
    return Status::success;
}

Status Server::wait(std::uint64_t ticket, std::uint64_t timeout_us, ServeOutcome &outcome,
                    bool &done) noexcept {
    Session &S = impl_->session;
    done = false;
    std::unique_lock<std::mutex> lock(S.mu);
    // Bounded at about 12 days so that the deadline cannot overflow.
    const auto limit = std::chrono::microseconds(std::min<std::uint64_t>(timeout_us, 1ull << 40));
    const bool settled = S.completed.wait_for(lock, limit, [&] {
        const auto it = S.tickets.find(ticket);
        return it == S.tickets.end() || it->second.done || S.failure != Status::success;
    });
    const auto it = S.tickets.find(ticket);
    if (it == S.tickets.end()) {
        return Status::invalid_argument;
    }
    if (it->second.done) {
        outcome = it->second.outcome;
        done = true;
        return Status::success;
    }
    return settled ? S.failure : Status::success;
}

Status Server::release(std::uint64_t ticket) noexcept {
    Session &S = impl_->session;
    {
        std::lock_guard<std::mutex> lock(S.mu);
        const auto it = S.tickets.find(ticket);
        if (it == S.tickets.end() || !it->second.done) {
            return Status::invalid_argument;
        }
        if (it->second.placed) {
            S.ring->release(it->second.seq);
        }
        S.tickets.erase(it);
    }
    S.wake.notify_one(); // output memory came back: a stalled request may fit now
    return Status::success;
}

Status Server::stop() noexcept {
    Impl &s = *impl_;
    Session &S = s.session;
    {
        std::lock_guard<std::mutex> lock(S.mu);
        if (!S.running) {
            return Status::invalid_argument;
        }
    }
    s.end_session();
    std::lock_guard<std::mutex> lock(S.mu);
    S.running = false;
    S.stopping = false;
    return S.failure;
}

// Gives every queued request the final status `status` (no output). Called with the lock held.
void Server::Impl::settle_queued(Status status) {
    for (const std::uint64_t id : session.queue) {
        Ticket &t = session.tickets.at(id);
        t.outcome.result.status = status;
        t.outcome.result.bytes_written = 0;
        t.done = true;
    }
    session.queue.clear();
}

void Server::Impl::session_loop() {
    Session &S = session;
    const bool device_ok = cudaSetDevice(device) == cudaSuccess;
    std::unique_lock<std::mutex> lock(S.mu);
    if (!device_ok) {
        S.failure = Status::cuda_error;
    }
    tsk_serve_batch batch;
    const std::uint32_t limit = options.max_batch;
    while (S.failure == Status::success) {
        // 1. Completions: the batch's records were copied to pinned memory in stream order.
        bool busy = false, finished = false;
        for (std::size_t k = 0; k < slots.size(); ++k) {
            Slot &slot = slots[k];
            if (!slot.busy) continue;
            const cudaError_t q = cudaEventQuery(slot.done);
            if (q == cudaErrorNotReady) {
                busy = true;
                continue;
            }
            if (q != cudaSuccess) {
                S.failure = detail::cuda_failure("serving batch", q);
                break;
            }
            const Clock::time_point now = Clock::now();
            const tsk_result *rec = S.host_records + k * limit;
            const std::vector<std::uint64_t> &ids = S.launched[k];
            for (std::size_t j = 0; j < ids.size(); ++j) {
                Ticket &t = S.tickets.at(ids[j]);
                t.outcome.result.status = static_cast<Status>(rec[j].status);
                t.outcome.result.bytes_written = rec[j].bytes_written;
                t.outcome.latency_us = micros(t.submitted, now);
                t.done = true;
            }
            S.launched[k].clear();
            slot.busy = false;
            finished = true;
        }
        if (finished) {
            S.completed.notify_all();
        }
        if (S.failure != Status::success) break;
        // 2. Admission, in submission order, while the pool has room; then one launch.
        std::size_t free_slot = slots.size();
        for (std::size_t k = 0; k < slots.size(); ++k) {
            if (!slots[k].busy) {
                free_slot = k;
                break;
            }
        }
        bool stalled = false;
        if (free_slot < slots.size() && !S.queue.empty()) {
            std::uint32_t n = 0;
            std::uint64_t ntasks = 0;
            std::vector<std::uint64_t> &ids = S.launched[free_slot];
            while (!S.queue.empty() && n < limit) {
                Ticket &t = S.tickets.at(S.queue.front());
                if (ntasks + t.tiles > options.max_batch_tiles && n != 0) break;
                std::uint64_t offset = 0;
                if (!S.ring->alloc(t.bytes, offset, t.seq)) {
                    stalled = true;
                    break;
                }
                t.placed = true;
                t.outcome.output_offset = offset;
                fill_record(batch.requests[n], t.request, archives[t.request.archive],
                            reinterpret_cast<std::uint64_t>(pool) + offset,
                            t.outcome.output_pitch);
                ntasks += t.tiles;
                batch.requests[n].task_end = static_cast<std::uint32_t>(ntasks);
                ids.push_back(S.queue.front());
                S.queue.pop_front();
                ++n;
            }
            if (n != 0) {
                batch.count = n;
                batch.ntasks = static_cast<std::uint32_t>(ntasks);
                Slot &slot = slots[free_slot];
                tsk_result *dev = S.device_records + free_slot * limit;
                const int e = tsk_serve_launch(&batch, dev_archives, dev_rows, dev, grid,
                                               all_u16 ? 1 : 0, slot.stream);
                if (e != 0 ||
                    cudaMemcpyAsync(S.host_records + free_slot * limit, dev,
                                    n * sizeof(tsk_result), cudaMemcpyDeviceToHost,
                                    slot.stream) != cudaSuccess ||
                    cudaEventRecord(slot.done, slot.stream) != cudaSuccess) {
                    S.failure = detail::cuda_failure("serving launch", static_cast<cudaError_t>(e));
                    break;
                }
                const Clock::time_point at = Clock::now();
                for (const std::uint64_t id : ids) {
                    Ticket &t = S.tickets.at(id);
                    t.outcome.queued_us = micros(t.submitted, at);
                    t.outcome.batch_size = n;
                }
                slot.busy = true;
                busy = true;
            }
        }
        if (S.stopping && !busy && (S.queue.empty() || stalled)) {
            // Requests that cannot fit while the outputs before them are held stay unserved.
            settle_queued(Status::resource_limit);
            S.completed.notify_all();
            break;
        }
        if (busy) {
            // Poll the in-flight launches without holding the lock.
            lock.unlock();
            std::this_thread::yield();
            lock.lock();
        } else if (S.queue.empty() || stalled) {
            // Idle until a submit, a release or stop (or, at the latest, a millisecond).
            S.wake.wait_for(lock, std::chrono::milliseconds(1));
        }
    }
    if (S.failure != Status::success) {
        lock.unlock();
        for (Slot &slot : slots) {
            if (slot.busy) {
                cudaEventSynchronize(slot.done);
                slot.busy = false;
            }
        }
        lock.lock();
        for (std::vector<std::uint64_t> &ids : S.launched) {
            for (const std::uint64_t id : ids) {
                Ticket &t = S.tickets.at(id);
                t.outcome.result.status = S.failure;
                t.done = true;
            }
            ids.clear();
        }
        settle_queued(S.failure);
        S.completed.notify_all();
    }
}

} // namespace tilestream::cuda
