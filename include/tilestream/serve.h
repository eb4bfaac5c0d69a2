#pragma once
// ROI serving over resident archives. This is an extension: the reference has no serving API.
//
// Archives stay in device memory with device tile tables built once (add_archive + seal).
// Requests are ROIs of one archive, plain or with fused scalar calibration. They arrive over
// time (ServeRequest::arrival_us) and are admitted in arrival order while the output pool has
// room for their pixels. The server then batches every admitted request that has arrived into
// one launch of the persistent decoder. The kernel expands each request's ROI into tile tasks
// itself, so a batch uploads nothing: its request records travel in the launch's parameter
// block. Up to max_inflight batches run on the GPU at once, one stream each. Requests that
// arrive while batches are running start on a free stream as soon as pool memory allows, so
// their work overlaps on the device (continuous batching).
//
// Requests can also be submitted while the server runs (start, submit, wait, release, stop):
// the same loop then serves them from a thread of its own as they come.
//
// The serial mode is the one-request-at-a-time baseline through the reference API:
// prepare_batch, then decode_roi_async or decode_calibrate_async, then a synchronize, per
// request.
#include <tilestream/api.h>
#include <tilestream/cuda.h>

#include <cstdint>
#include <memory>

namespace tilestream::cuda {

struct ServeRequest {
    std::uint32_t archive = 0; // id from Server::add_archive
    Roi roi;
    std::uint32_t calibrated = 0; // nonzero: FP32 output RN(RN(x - offset) * gain)
    float offset = 0.0F;
    float gain = 1.0F;
    double arrival_us = 0.0; // arrival time after the start of Server::run; non-decreasing
};

struct ServeOptions {
    std::uint64_t output_pool_bytes = 1ull << 30; // device memory for request outputs
    std::uint32_t max_batch = 48;                 // requests per launch (at most 48)
    std::uint32_t max_inflight = 4;               // batches on the GPU at once (at most 16)
    std::uint64_t max_batch_tiles = 1u << 22;     // tile tasks per launch
    std::uint32_t retain_outputs = 0; // nonzero: outputs stay valid until the run ends
    std::uint32_t serial = 0;         // nonzero: one request at a time through the plan API
};

struct ServeStats {
    double wall_us = 0;        // start of the run to the last completion
    double throughput_rps = 0; // completed requests per second of wall time
    double decoded_gbs = 0;    // output bytes per second of wall time
    double p50_us = 0, p90_us = 0, p99_us = 0, max_us = 0, mean_us = 0; // latency, nearest rank
    std::uint64_t completed = 0;   // requests that ran (any status)
    std::uint64_t rejected = 0;    // requests refused on the host (invalid or oversize)
    std::uint64_t batches = 0;     // launches
    double mean_batch = 0;         // requests per launch
    std::uint64_t max_inflight = 0; // most batches seen on the GPU at once
    std::uint64_t stalls = 0;      // requests that had arrived but waited for pool memory
    std::uint64_t tiles = 0;       // tile tasks decoded
    std::uint64_t output_bytes = 0;
};

// Per-request outcome of a run, in request order.
struct ServeOutcome {
    double latency_us = 0;  // completion seen by the server minus arrival
    double queued_us = 0;   // launch minus arrival
    std::uint64_t output_offset = 0; // pixel (0, 0) of the request's output within the pool
    std::uint64_t output_pitch = 0;  // bytes per output row (a multiple of 16)
    std::uint32_t batch_size = 0;    // requests in the launch that served this one
    DeviceResult result;    // the device record, or the host's refusal
};

class Server {
  public:
    ~Server();
    Server(const Server &) = delete;
    Server &operator=(const Server &) = delete;

    // A server on the current device; the output pool, streams and events are created here.
    [[nodiscard]] static Status create(const ServeOptions &options,
                                       std::unique_ptr<Server> &out) noexcept;
    // Registers a resident archive: the device bytes of the complete file and its parsed
    // metadata. Every tile is validated here once. Both must outlive the server.
    [[nodiscard]] Status add_archive(ConstBytes device_bytes, const ImageMetadata &metadata,
                                     std::uint32_t &id) noexcept;
    // Uploads the tile tables of the registered archives; required before run().
    [[nodiscard]] Status seal() noexcept;
    // Serves the requests in arrival order. outcomes (count entries) and stats are filled in.
    // Refused requests (unknown archive, ROI outside it, output larger than the pool) report
    // their status in the outcome and do not stop the run. One run at a time per server.
    [[nodiscard]] Status run(const ServeRequest *requests, std::uint64_t count,
                             ServeOutcome *outcomes, ServeStats &stats) noexcept;
    // The output pool (device memory).
    [[nodiscard]] MutableBytes pool() const noexcept;

    // ---- request sessions: requests submitted while the server runs ----
    // start() launches the serving loop on a thread of its own: from then on, requests
    // submitted from any thread are admitted by output-pool memory, batched into launches and
    // overlapped on the GPU exactly as in run(). A request's output stays in the pool until the
    // caller releases it, so results can be read at leisure. At most `max_outstanding` requests
    // (submitted and not yet released) at a time. run() is not available while started.
    [[nodiscard]] Status start(std::uint32_t max_outstanding = 4096) noexcept;
    // Queues a request (arrival_us is ignored: it arrives now). ticket identifies it. Refused
    // requests (unknown archive, ROI outside it, output larger than the pool) return their
    // status here and take no ticket; resource_limit when too many are outstanding.
    [[nodiscard]] Status submit(const ServeRequest &request, std::uint64_t &ticket) noexcept;
    // Waits at most timeout_us for the request to complete; done tells whether it has. When
    // done, outcome holds its result, output place and latency (submit to completion).
    [[nodiscard]] Status wait(std::uint64_t ticket, std::uint64_t timeout_us,
                              ServeOutcome &outcome, bool &done) noexcept;
    // Gives the request's output memory back to the pool; the ticket is then unknown.
    // invalid_argument for an unknown ticket or one that has not completed.
    [[nodiscard]] Status release(std::uint64_t ticket) noexcept;
    // Serves what was submitted, then ends the loop (unreleased outputs stay readable until the
    // server is destroyed or started again).
    [[nodiscard]] Status stop() noexcept;

    struct Impl;

  private:
    std::unique_ptr<Impl> impl_;
    explicit Server(std::unique_ptr<Impl> impl) noexcept;
};

} // namespace tilestream::cuda
