"""Mixed batches: uint16 and FP32 archives of uneven sizes and all three tile geometries,
whole-image, ROI, calibrated and trusted (encoder-output) items in ONE persistent kernel,
replayed as a CUDA graph, with and without the autotuner. Every output is compared with the
oracle, and every result record with the single-item executors' contract."""
import numpy as np
import pytest

import oracle
from support import SENTINEL, crop, device_bytes, host, logical, parsed_source, to_device, Run
from tilestream_b200 import api, cuda, workloads
from tilestream_b200.api import BatchItem, CompressedInput, ConstBytes, Status, TileShape

pytestmark = pytest.mark.gpu


def build_items(o, seeds):
    """One item per seeded case, cycling through decompress, decode_roi and decode_calibrate."""
    items, keep, checks = [], [], []
    for n, seed in enumerate(seeds):
        c = o.case(seed)
        s = oracle.SAMPLE[c["type"]]
        w, h = c["width"], c["height"]
        file = o.compress(c["bytes"], c["type"], w, h, c["pitch"], c["tile"])
        src, meta, dev = parsed_source(file)
        keep += [meta, dev]
        kind = n % 3
        roi = c["roi"] if kind else (0, 0, w, h)
        rx, ry, rw, rh = roi
        item = BatchItem()
        item.compressed_input = src
        if kind == 2:
            out_pitch = rw * 4 + 8
            out = device_bytes(out_pitch * rh)
            item.output = api.view(out, 2, rw, rh, out_pitch, out.numel())
            item.roi = api.Roi(*roi)
            item.calibration.offset.scalar = 100.0
            item.calibration.gain.scalar = 1.05
            op = cuda.Operation.decode_calibrate
            region = crop(c["bytes"], c["pitch"], s, roi).view(
                np.uint16 if s == 2 else np.uint32).reshape(rh, rw)
            want = o.calibrate_image(region, 100.0, 1.05).view(np.uint8).reshape(rh, rw * 4)
            checks.append((out, out_pitch, rw * 4, rh, want, rw * rh * 4))
        else:
            out_pitch = rw * s + 2 * s
            out = device_bytes(out_pitch * rh)
            item.output = api.view(out, c["type"], rw, rh, out_pitch, out.numel())
            op = cuda.Operation.decompress
            if kind == 1:
                item.roi = api.Roi(*roi)
                op = cuda.Operation.decode_roi
            want = crop(c["bytes"], c["pitch"], s, roi).reshape(rh, rw * s)
            checks.append((out, out_pitch, rw * s, rh, want, rw * rh * s))
        keep.append(out)
        items.append((op, item))
    return items, keep, checks


def verify(checks, results):
    raw = host(results).view(np.uint64).reshape(-1, 2)
    for k, (out, pitch, row_bytes, rh, want, nbytes) in enumerate(checks):
        assert int(raw[k, 0]) == 0 and int(raw[k, 1]) == nbytes, k
        got = host(out)[:pitch * rh].reshape(rh, pitch)
        rows = np.ascontiguousarray(got[:, :row_bytes])
        if nbytes == rh * row_bytes and (k % 3) == 2:
            # Calibrated FP32: bit-exact except NaN payloads (NaNs compare by class).
            a, b = rows.view(np.float32), np.ascontiguousarray(want).view(np.float32)
            assert np.all((a.view(np.uint32) == b.view(np.uint32)) |
                          (np.isnan(a) & np.isnan(b))), k
        else:
            assert np.array_equal(rows, want), k
        assert np.all(got[:, row_bytes:] == SENTINEL), k


@pytest.mark.parametrize("graph,autotune", [(True, False), (False, False), (True, True)])
def test_mixed_batch_matches_oracle(cuda_ready, oracle_lib, graph, autotune):
    torch = cuda_ready
    seeds = list(range(13002000, 13002000 + 90))
    items, keep, checks = build_items(oracle_lib, seeds)
    results = device_bytes(16 * len(items), fill=0xFF)
    stream = torch.cuda.current_stream()
    st, batch = cuda.prepare_mixed_batch(items, results, stream, graph=graph, autotune=autotune)
    assert st == Status.success, st
    stats = batch.stats()
    assert stats["graph"] == graph
    for _ in range(2):  # executions repeat on the same bound buffers
        assert batch.run(stream) == Status.success
        torch.cuda.synchronize()
        verify(checks, results)


def test_mixed_batch_with_trusted_items(cuda_ready, oracle_lib):
    """Encoder output decoded on the device in the same batch as parsed archives."""
    torch = cuda_ready
    stream = torch.cuda.current_stream()
    frame = workloads.detector_frame(700, 300, seed=71)
    dev_in = to_device(frame)
    st, bound = api.compress_bound(api.image_spec(1, 700, 300), TileShape(64, 64))
    archive = device_bytes(bound)
    enc = BatchItem()
    enc.input = api.const_view(dev_in, 1, 700, 300, 1400, dev_in.numel())
    enc.compressed_output = api.MutableBytes(archive.data_ptr(), bound)
    erun = Run(cuda.Operation.compress, [enc], tile=TileShape(64, 64), keep=[dev_in, archive])
    assert erun.execute(cuda.compress_async) == Status.success
    items, keep, checks = build_items(oracle_lib, list(range(13003000, 13003012)))
    src = CompressedInput()
    src.bytes = ConstBytes(archive.data_ptr(), bound)
    src.encoder_result = erun.results.data_ptr()
    src.trusted_image = api.image_spec(1, 700, 300)
    src.trusted_tile = TileShape(64, 64)
    out = device_bytes(700 * 300 * 2)
    item = BatchItem()
    item.compressed_input = src
    item.output = api.view(out, 1, 700, 300, 1400, out.numel())
    items.append((cuda.Operation.decompress, item))
    checks.append((out, 1400, 1400, 300, frame.view(np.uint8).reshape(300, 1400), 700 * 300 * 2))
    results = device_bytes(16 * len(items), fill=0xFF)
    st, batch = cuda.prepare_mixed_batch(items, results, stream)
    assert st == Status.success
    assert batch.run(stream) == Status.success
    torch.cuda.synchronize()
    verify(checks, results)


def test_mixed_batch_validation(cuda_ready, oracle_lib):
    torch = cuda_ready
    stream = torch.cuda.current_stream()
    items, keep, checks = build_items(oracle_lib, [13004000, 13004001])
    results = device_bytes(16 * len(items))
    bad = [(cuda.Operation.compress, items[0][1])]
    assert cuda.prepare_mixed_batch(bad, results, stream)[0] == Status.invalid_argument
    assert cuda.prepare_mixed_batch(items, device_bytes(16), stream)[0] == Status.buffer_too_small
    # Results overlapping an output are rejected.
    out = items[0][1].output
    overlap = api.ResultBuffer(out.data, 2)
    assert cuda.prepare_mixed_batch(items, overlap, stream)[0] == Status.invalid_argument
    st, empty = cuda.prepare_mixed_batch([], results, stream)
    assert st == Status.success and empty.run(stream) == Status.success


def plain_items(o, seeds, f32):
    """Decompress and decode_roi items only (no calibration), uint16 only or uint16 + FP32."""
    picked = [s for s in seeds if f32 or o.case(s)["type"] == 1]
    items, keep, checks = build_items(o, picked)
    kept = [(it, c) for it, c in zip(items, checks) if it[0] != cuda.Operation.decode_calibrate]
    return [it for it, _ in kept], keep, [c for _, c in kept]


def verify_plain(checks, results):
    raw = host(results).view(np.uint64).reshape(-1, 2)
    for k, (out, pitch, row_bytes, rh, want, nbytes) in enumerate(checks):
        assert int(raw[k, 0]) == 0 and int(raw[k, 1]) == nbytes, k
        got = host(out)[:pitch * rh].reshape(rh, pitch)
        assert np.array_equal(np.ascontiguousarray(got[:, :row_bytes]), want), k
        assert np.all(got[:, row_bytes:] == SENTINEL), k


@pytest.mark.parametrize("f32", [False, True])
def test_every_kernel_shape_matches_oracle(cuda_ready, oracle_lib, f32):
    """Each kernel shape (MixedOptions.shape), forced in turn on plain batches - uint16 only, and
    uint16 with FP32 - decodes every item to the oracle's words."""
    torch = cuda_ready
    stream = torch.cuda.current_stream()
    items, keep, checks = plain_items(oracle_lib, list(range(13005000, 13005060)), f32)
    assert any(op == cuda.Operation.decode_roi for op, _ in items)
    for shape in range(cuda.decode_shape_count()):
        for graph in (True, False):
            results = device_bytes(16 * len(items), fill=0xFF)
            for out, pitch, row_bytes, rh, want, nbytes in checks:
                out.fill_(SENTINEL)
            st, batch = cuda.prepare_mixed_batch(items, results, stream, shape=shape, graph=graph)
            assert st == Status.success, (shape, st)
            assert batch.stats()["shape"] == shape
            # Twice: shapes with the device work queue clear its counter before every launch.
            assert batch.run(stream) == Status.success
            assert batch.run(stream) == Status.success
            torch.cuda.synchronize()
            verify_plain(checks, results)
    st, _ = cuda.prepare_mixed_batch(items, device_bytes(16 * len(items)), stream,
                                     shape=cuda.decode_shape_count())
    assert st == Status.invalid_argument
