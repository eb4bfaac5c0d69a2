"""ROI serving over resident archives: every request's output, served in a mix of co-arriving
requests with continuous batching, equals the oracle's crop (or calibrated crop) and the same
request served alone; the one-request-at-a-time plan path agrees; a small output pool forces
admission stalls without changing any result; refusals are per request. Sessions: requests
submitted by two producer threads while the server runs, waited for (bounded) and released by a
consumer thread, equal the oracle and the same request served alone; releases admit stalled
requests, and stop settles what cannot be placed."""
import numpy as np
import pytest

from support import read_device, to_device
from tilestream_b200 import api, cuda, workloads
from tilestream_b200.api import ConstBytes, Status

pytestmark = pytest.mark.gpu

# uint16 archives of three tile geometries and one FP32 archive, uneven sizes.
ARCHIVES = [("u16", 1000, 700, (64, 64), 31), ("u16", 777, 513, (128, 32), 32),
            ("u16", 900, 450, (256, 16), 33), ("f32", 600, 500, (64, 64), 34)]


class Fixture:
    def __init__(self, o):
        self.pixels, self.files = [], []
        for kind, w, h, tile, seed in ARCHIVES:
            frame = (workloads.detector_frame(w, h, seed) if kind == "u16"
                     else workloads.field_frame(w, h, seed))
            self.pixels.append(frame)
            self.files.append(o.compress_image(frame, tile))

    def server(self, **options):
        srv = cuda.Server(**options)
        for file in self.files:
            st, meta = api.parse_metadata(file)
            assert st == Status.success
            dev = to_device(np.frombuffer(file, np.uint8))
            st, _ = srv.add_archive(ConstBytes(dev.data_ptr(), len(file)), meta, owner=dev)
            assert st == Status.success
        assert srv.seal() == Status.success
        return srv


@pytest.fixture(scope="module")
def fx(oracle_lib):
    return Fixture(oracle_lib)


def stream_of(n, seed, rate=40000.0, max_side=700):
    """Requests over the four archives, ROIs fitted to each archive."""
    rng = np.random.Generator(np.random.PCG64(seed))
    reqs = (cuda.N.ServeRequest * n)()
    t = 0.0
    for i in range(n):
        a = int(rng.integers(0, len(ARCHIVES)))
        _, w, h, _, _ = ARCHIVES[a]
        rw = int(min(w, np.exp(rng.uniform(np.log(1), np.log(max_side)))))
        rh = int(min(h, np.exp(rng.uniform(np.log(1), np.log(max_side)))))
        rw, rh = max(rw, 1), max(rh, 1)
        x = int(rng.integers(0, w - rw + 1))
        y = int(rng.integers(0, h - rh + 1))
        t += float(rng.exponential(1e6 / rate))
        r = reqs[i]
        r.archive = a
        r.roi = api.Roi(x, y, rw, rh)
        r.calibrated = 1 if rng.random() < 0.4 else 0
        r.offset, r.gain = 100.0, 1.05
        r.arrival_us = t
    return reqs


def expected(o, fx, r):
    """The oracle's answer for one request: bytes of the (h, w * sample) region."""
    frame = fx.pixels[r.archive]
    x, y, w, h = r.roi.x, r.roi.y, r.roi.width, r.roi.height
    region = np.ascontiguousarray(frame[y:y + h, x:x + w])
    if r.calibrated:
        return o.calibrate_image(region, r.offset, r.gain).view(np.uint8).reshape(h, w * 4), True
    return region.view(np.uint8).reshape(h, -1), False


def output_of(pool_host, outcome, r, fx):
    sample = 4 if (r.calibrated or ARCHIVES[r.archive][0] == "f32") else 2
    w, h = r.roi.width, r.roi.height
    pitch = outcome.output_pitch
    assert pitch % 16 == 0 and pitch >= w * sample
    start = outcome.output_offset
    rows = pool_host[start:start + pitch * h].reshape(h, pitch)
    return np.ascontiguousarray(rows[:, :w * sample])


def same(got, want, float_words):
    if not float_words:
        return np.array_equal(got, want)
    a, b = got.view(np.float32), want.view(np.float32)
    return bool(np.all((a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))))


def check_outputs(o, fx, srv, reqs, outcomes, used):
    pool = read_device(srv.pool().data, used)
    outputs = []
    for i, r in enumerate(reqs):
        oc = outcomes[i]
        assert oc.result.status == 0, (i, oc.result.status)
        want, _ = expected(o, fx, r)
        assert oc.result.bytes_written == want.size, i
        got = output_of(pool, oc, r, fx)
        assert same(got, want, r.calibrated != 0), i
        outputs.append(got)
    return outputs


def pool_need(reqs):
    total = 0
    for r in reqs:
        s = 4 if (r.calibrated or ARCHIVES[r.archive][0] == "f32") else 2
        total += ((r.roi.width * s + 15) // 16 * 16 * r.roi.height + 255) // 256 * 256
    return total


def test_mix_equals_oracle_and_alone(cuda_ready, oracle_lib, fx):
    reqs = stream_of(160, seed=5001)
    need = pool_need(reqs)
    srv = fx.server(pool_bytes=need, retain_outputs=True, max_inflight=4)
    st, outcomes, stats = srv.run(reqs)
    assert st == Status.success
    assert stats.completed == len(reqs) and stats.rejected == 0
    assert stats.batches >= 1 and stats.tiles > 0
    mixed = check_outputs(oracle_lib, fx, srv, reqs, outcomes, need)
    # Alone: each request on its own, arriving at once.
    for i in range(0, len(reqs), 7):
        one = (cuda.N.ServeRequest * 1)(reqs[i])
        one[0].arrival_us = 0.0
        st, oc, s1 = srv.run(one)
        assert st == Status.success and s1.batches == 1 and oc[0].batch_size == 1
        assert oc[0].output_offset == 0
        alone = output_of(read_device(srv.pool().data, oc[0].output_pitch * one[0].roi.height),
                          oc[0], one[0], fx)
        assert same(alone, mixed[i], one[0].calibrated != 0), i


def test_burst_batches_and_overlaps(cuda_ready, oracle_lib, fx):
    """All requests arrive at once: they are batched (several per launch) and several
    launches run at once."""
    reqs = stream_of(120, seed=5002)
    for r in reqs:
        r.arrival_us = 0.0
    need = pool_need(reqs)
    srv = fx.server(pool_bytes=need, retain_outputs=True, max_batch=16, max_inflight=3)
    st, outcomes, stats = srv.run(reqs)
    assert st == Status.success
    assert stats.mean_batch > 1.0 and stats.max_inflight >= 2
    assert max(outcomes[i].batch_size for i in range(len(reqs))) <= 16
    check_outputs(oracle_lib, fx, srv, reqs, outcomes, need)


def test_small_pool_stalls_admission(cuda_ready, oracle_lib, fx):
    """A burst into a pool of two of the largest outputs: arrived requests wait for memory,
    and every record still reports success with its byte count."""
    reqs = stream_of(150, seed=5003)
    for r in reqs:
        r.arrival_us = 0.0
    biggest = max(pool_need([r]) for r in reqs)
    assert pool_need(reqs) > 2 * biggest
    srv = fx.server(pool_bytes=2 * biggest, max_inflight=4)
    st, outcomes, stats = srv.run(reqs)
    assert st == Status.success
    assert stats.stalls > 0 and stats.completed == len(reqs)
    for i, r in enumerate(reqs):
        want, _ = expected(oracle_lib, fx, r)
        assert outcomes[i].result.status == 0 and outcomes[i].result.bytes_written == want.size
    # Nothing was admitted after the last launch (the last batch_size requests): its outputs
    # are still in the pool.
    n = outcomes[len(reqs) - 1].batch_size
    last = range(len(reqs) - n, len(reqs))
    pool = read_device(srv.pool().data, 2 * biggest)
    for i in last:
        want, _ = expected(oracle_lib, fx, reqs[i])
        assert same(output_of(pool, outcomes[i], reqs[i], fx), want, reqs[i].calibrated != 0)


def test_serial_plan_path_agrees(cuda_ready, oracle_lib, fx):
    reqs = stream_of(40, seed=5004)
    need = pool_need(reqs)
    srv = fx.server(pool_bytes=need, retain_outputs=True, serial=True)
    st, outcomes, stats = srv.run(reqs)
    assert st == Status.success and stats.batches == len(reqs) and stats.mean_batch == 1.0
    check_outputs(oracle_lib, fx, srv, reqs, outcomes, need)


def test_refusals_are_per_request(cuda_ready, oracle_lib, fx):
    reqs = stream_of(12, seed=5005, max_side=64)
    bad = {3: Status.invalid_argument, 6: Status.invalid_roi, 9: Status.buffer_too_small}
    reqs[3].archive = 99
    reqs[6].roi = api.Roi(990, 0, 20, 10)  # archive 0 is 1000 wide: 990 + 20 is outside
    reqs[6].archive = 0
    good = [r for i, r in enumerate(reqs) if i not in bad]
    need = pool_need(good)
    reqs[9].archive = 0
    reqs[9].roi = api.Roi(0, 0, 1000, 700)
    reqs[9].calibrated = 1  # 2.8 MB: larger than the 1 MiB pool below
    assert need <= 1 << 20
    srv = fx.server(pool_bytes=1 << 20, retain_outputs=True)
    st, outcomes, stats = srv.run(reqs)
    assert st == Status.success and stats.rejected == 3
    for i, r in enumerate(reqs):
        if i in bad:
            assert outcomes[i].result.status == int(bad[i]) and outcomes[i].batch_size == 0
        else:
            want, _ = expected(oracle_lib, fx, r)
            assert outcomes[i].result.status == 0 and outcomes[i].result.bytes_written == want.size


def test_host_validation(cuda_ready, oracle_lib, fx):
    srv = cuda.Server(pool_bytes=1 << 20)
    reqs = stream_of(2, seed=5006)
    assert srv.run(reqs)[0] == Status.invalid_argument  # not sealed
    assert srv.seal() == Status.invalid_argument        # nothing to serve
    sealed = fx.server(pool_bytes=1 << 24)
    reqs[1].arrival_us = reqs[0].arrival_us - 1.0
    assert sealed.run(reqs)[0] == Status.invalid_argument  # arrivals out of order
    st, meta = api.parse_metadata(fx.files[0])
    dev = to_device(np.frombuffer(fx.files[0], np.uint8))
    assert sealed.add_archive(ConstBytes(dev.data_ptr(), len(fx.files[0])), meta)[0] == \
        Status.invalid_argument  # sealed
    # A tile whose length exceeds its raw size is refused when the archive is added.
    tiles = meta.tiles.copy()
    tiles[0]["length"] = 1 << 20
    st, bad = api.ImageMetadata.create(meta.image, meta.tile, meta.file_bytes, tiles,
                                       meta.segments)
    assert st == Status.success
    fresh = cuda.Server(pool_bytes=1 << 20)
    assert fresh.add_archive(ConstBytes(dev.data_ptr(), len(fx.files[0])), bad)[0] == \
        Status.malformed_data
    with pytest.raises(RuntimeError):
        cuda.Server(max_batch=49)


# ---- sessions: requests submitted while the server runs --------------------------------------

def _submit_bounded(srv, r, seconds=20.0):
    """Submits r, retrying while too many requests are outstanding (bounded)."""
    import time
    end = time.monotonic() + seconds
    while True:
        st, ticket = srv.submit(r)
        if st != Status.resource_limit or time.monotonic() > end:
            return st, ticket
        time.sleep(0.001)


def _session_output(srv, outcome, r):
    sample = 4 if (r.calibrated or ARCHIVES[r.archive][0] == "f32") else 2
    rows = read_device(srv.pool().data + outcome.output_offset,
                       outcome.output_pitch * r.roi.height)
    rows = rows.reshape(r.roi.height, outcome.output_pitch)
    return np.ascontiguousarray(rows[:, :r.roi.width * sample])


def test_session_two_producers_one_consumer(cuda_ready, oracle_lib, fx):
    """Two producer threads submit interleaved halves of a request stream while one consumer
    waits (bounded), checks each output against the oracle and releases it. The pool holds
    four of the largest outputs, so admission also waits for releases. Afterwards the same
    requests served alone (run) give the same bytes."""
    import queue
    import threading
    reqs = stream_of(240, seed=5007)
    biggest = max(pool_need([r]) for r in reqs)
    srv = fx.server(pool_bytes=4 * biggest, max_batch=16, max_inflight=4)
    assert srv.submit(reqs[0])[0] == Status.invalid_argument  # not started
    assert srv.start(max_outstanding=32) == Status.success
    assert srv.run(reqs)[0] == Status.invalid_argument  # run() is closed while started
    handed = queue.Queue()
    errors = []

    def producer(part):
        for i in range(part, len(reqs), 2):
            st, ticket = _submit_bounded(srv, reqs[i])
            if st != Status.success:
                errors.append((i, st))
                handed.put(None)
                return
            handed.put((i, ticket))

    threads = [threading.Thread(target=producer, args=(p,)) for p in (0, 1)]
    for t in threads:
        t.start()
    got, batches = {}, []
    try:
        for _ in range(len(reqs)):
            item = handed.get(timeout=60)
            assert item is not None, errors
            i, ticket = item
            st, done, oc = srv.wait(ticket, timeout_us=10_000_000)
            assert st == Status.success and done, (i, st, done)
            assert oc.result.status == 0 and oc.batch_size >= 1, i
            want, _ = expected(oracle_lib, fx, reqs[i])
            assert oc.result.bytes_written == want.size, i
            out = _session_output(srv, oc, reqs[i])
            assert same(out, want, reqs[i].calibrated != 0), i
            got[i] = out
            batches.append(oc.batch_size)
            assert srv.release(ticket) == Status.success
            assert srv.release(ticket) == Status.invalid_argument  # released already
    finally:
        for t in threads:
            t.join(timeout=60)
        assert srv.stop() == Status.success
    assert not errors and len(got) == len(reqs)
    assert max(batches) > 1  # requests from both producers shared launches
    for i in range(0, len(reqs), 9):
        one = (cuda.N.ServeRequest * 1)(reqs[i])
        one[0].arrival_us = 0.0
        st, oc, _ = srv.run(one)
        assert st == Status.success and oc[0].batch_size == 1
        assert same(_session_output(srv, oc[0], one[0]), got[i], one[0].calibrated != 0), i


def test_session_release_admits_and_stop_settles(cuda_ready, oracle_lib, fx):
    """A pool with room for one output: the second request waits for the first's release (a
    bounded wait reports not done meanwhile); at stop, a request that cannot be placed while
    an output is held completes with resource_limit."""
    r = stream_of(1, seed=5008)[0]
    r.archive, r.roi, r.calibrated = 0, api.Roi(0, 0, 1000, 700), 0
    size = pool_need([r])
    srv = fx.server(pool_bytes=size)
    assert srv.start(max_outstanding=2) == Status.success
    st, a = srv.submit(r)
    assert st == Status.success
    st, b = srv.submit(r)
    assert st == Status.success
    assert srv.submit(r)[0] == Status.resource_limit  # two outstanding
    st, done, oa = srv.wait(a, timeout_us=10_000_000)
    assert st == Status.success and done and oa.result.status == 0
    want, _ = expected(oracle_lib, fx, r)
    assert np.array_equal(_session_output(srv, oa, r), want)
    st, done, _ = srv.wait(b, timeout_us=200_000)
    assert st == Status.success and not done  # held: a's output occupies the pool
    assert srv.release(b) == Status.invalid_argument  # not complete
    assert srv.release(a) == Status.success
    st, done, ob = srv.wait(b, timeout_us=10_000_000)
    assert st == Status.success and done and ob.result.status == 0
    assert np.array_equal(_session_output(srv, ob, r), want)
    # b's output is held: c cannot be placed, and stop settles it.
    st, c = srv.submit(r)
    assert st == Status.success
    assert srv.stop() == Status.success
    st, done, oc = srv.wait(c, timeout_us=0)
    assert st == Status.success and done
    assert oc.result.status == int(Status.resource_limit) and oc.result.bytes_written == 0
    assert srv.wait(12345, timeout_us=0)[0] == Status.invalid_argument  # unknown ticket
    assert srv.stop() == Status.invalid_argument  # not started
    # Started again: a fresh session over the same archives.
    assert srv.start() == Status.success
    st, d = srv.submit(r)
    st, done, od = srv.wait(d, timeout_us=10_000_000)
    assert st == Status.success and done and od.result.status == 0 and od.output_offset == 0
    assert srv.stop() == Status.success
