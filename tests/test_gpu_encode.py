"""GPU encoder parity: bitstreams byte-identical to the oracle's canonical encoding (golden files,
seeded cases, full-size frames, many-image batches), plus the trusted GPU round trip that decodes
the encoder's output without a host index (reference tests/cuda_encoder_test.cpp and
cuda_decoder_test.cpp:333-452)."""
import json
import os

import numpy as np
import pytest

import oracle
from support import SENTINEL, Run, device_bytes, host, logical, to_device
from tilestream_b200 import api, cuda, workloads
from tilestream_b200.api import BatchItem, CompressedInput, ConstBytes, Status, TileShape

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def read_hex(name):
    with open(os.path.join(GOLDEN, name + ".hex")) as f:
        return bytes(int(t, 16) for t in f.read().split())


def gpu_encode_many(images, tile=(128, 32), pitches=None):
    """images: list of (flat bytes, ptype, width, height, pitch). Returns (files, records)."""
    items, keep, outs = [], [], []
    for buf, ptype, w, h, pitch in images:
        dev = to_device(buf)
        st, bound = api.compress_bound(api.image_spec(ptype, w, h), TileShape(*tile))
        assert st == Status.success
        out = device_bytes(bound + 64)
        item = BatchItem()
        item.input = api.const_view(dev, ptype, w, h, pitch, dev.numel())
        item.compressed_output = api.MutableBytes(out.data_ptr(), bound)
        items.append(item)
        keep += [dev, out]
        outs.append((out, bound))
    run = Run(cuda.Operation.compress, items, tile=TileShape(*tile), keep=keep)
    assert run.status == Status.success, run.status
    assert run.execute(cuda.compress_async) == Status.success
    recs = run.records()
    files = []
    for (out, bound), rec in zip(outs, recs):
        data = host(out)
        assert rec[0] == 0 and rec[1] == 0 and rec[2] <= bound
        assert np.all(data[bound:] == SENTINEL)  # guard bytes after the bound
        files.append(data[:rec[2]].tobytes())
    return files, recs


def test_golden_files_encode(cuda_ready):
    cases = json.load(open(os.path.join(GOLDEN, "cases.json")))
    for name, c in cases.items():
        dtype = np.uint16 if c["type"] == 1 else np.uint32
        px = np.array(c["pixels"], dtype=dtype)
        files, _ = gpu_encode_many([(px, c["type"], c["width"], c["height"],
                                     c["width"] * px.itemsize)])
        assert files[0] == read_hex(name), name


@pytest.mark.parametrize("first", [13000000, 13003000])
def test_robustness_cases_byte_identical(cuda_ready, oracle_lib, first):
    o = oracle_lib
    for ptype_parity in (0, 1):
        for tile_index, tile in enumerate(api.TILE_SHAPES):
            seeds = [first + 6 * k + ptype_parity + 2 * tile_index for k in range(40)]
            cases = [o.case(s) for s in seeds]
            images = [(c["bytes"], c["type"], c["width"], c["height"], c["pitch"]) for c in cases]
            files, _ = gpu_encode_many(images, tile)
            for c, f in zip(cases, files):
                want = o.compress(c["bytes"], c["type"], c["width"], c["height"], c["pitch"], tile)
                assert f == want, c["seed"]


@pytest.mark.parametrize("tile", api.TILE_SHAPES)
def test_detector_frame_byte_identical(cuda_ready, oracle_lib, tile):
    frame = workloads.detector_frame(4096, 4096, seed=2)
    files, _ = gpu_encode_many([(frame, 1, 4096, 4096, 8192)], tile)
    assert files[0] == oracle_lib.compress_image(frame, tile)


def test_field_frame_byte_identical(cuda_ready, oracle_lib):
    frame = workloads.field_frame(2048, 1500, seed=3)
    files, _ = gpu_encode_many([(frame, 2, 2048, 1500, 8192)])
    assert files[0] == oracle_lib.compress_image(frame, (128, 32))


def test_many_small_images(cuda_ready, oracle_lib):
    rng = np.random.default_rng(3)
    images, arrays = [], []
    for k in range(300):
        w, h = int(rng.integers(1, 200)), int(rng.integers(1, 90))
        img = oracle_lib.fill(1, w, h, int(rng.integers(0, 8)), 1000 + k).view(np.uint16)
        arrays.append(img.reshape(h, w))
        images.append((img, 1, w, h, w * 2))
    files, _ = gpu_encode_many(images, (64, 64))
    for img, f in zip(arrays, files):
        assert f == oracle_lib.compress_image(img, (64, 64))


def test_trusted_round_trip(cuda_ready, oracle_lib):
    """Encoder output decoded on the device with no host index (whole image and ROI)."""
    frames = [workloads.detector_frame(1500, 900, seed=31), workloads.detector_frame(257, 4097, 32)]
    for frame in frames:
        h, w = frame.shape
        dev_in = to_device(frame)
        st, bound = api.compress_bound(api.image_spec(1, w, h), TileShape())
        archive = device_bytes(bound)
        enc = BatchItem()
        enc.input = api.const_view(dev_in, 1, w, h, w * 2, dev_in.numel())
        enc.compressed_output = api.MutableBytes(archive.data_ptr(), bound)
        erun = Run(cuda.Operation.compress, [enc], keep=[dev_in, archive])
        assert erun.status == Status.success
        assert erun.execute(cuda.compress_async) == Status.success
        for roi in (None, (17, 33, w - 40, h - 70)):
            src = CompressedInput()
            src.bytes = ConstBytes(archive.data_ptr(), bound)
            src.encoder_result = erun.results.data_ptr()
            src.trusted_image = api.image_spec(1, w, h)
            src.trusted_tile = TileShape()
            rw, rh = (w, h) if roi is None else roi[2:]
            out = device_bytes(rw * rh * 2)
            item = BatchItem()
            item.compressed_input = src
            item.output = api.view(out, 1, rw, rh, rw * 2, out.numel())
            op = cuda.Operation.decompress
            if roi is not None:
                item.roi = api.Roi(*roi)
                op = cuda.Operation.decode_roi
            drun = Run(op, [item], keep=[out])
            assert drun.status == Status.success
            ex = cuda.decompress_async if roi is None else cuda.decode_roi_async
            assert drun.execute(ex) == Status.success
            assert drun.records()[0] == (0, 0, rw * rh * 2)
            want = frame if roi is None else frame[roi[1]:roi[1] + rh, roi[0]:roi[0] + rw]
            assert np.array_equal(host(out).view(np.uint16).reshape(rh, rw), want)
        # The encoded bytes are the oracle's.
        assert host(archive)[:erun.records()[0][2]].tobytes() == oracle_lib.compress_image(frame)


def test_trusted_corrupt_index_is_malformed(cuda_ready, oracle_lib):
    """A corrupted index entry of an encoder output is reported as malformed_data with zero
    bytes, not read (reference cuda_decoder_test.cpp:431-452)."""
    frame = workloads.detector_frame(300, 100, seed=41)
    file = bytearray(oracle_lib.compress_image(frame))
    file[64 + 32 * 2 + 4] ^= 0xFF  # width of tile 2
    st, bound = api.compress_bound(api.image_spec(1, 300, 100), TileShape())
    padded = np.zeros(bound, dtype=np.uint8)
    padded[:len(file)] = np.frombuffer(bytes(file), dtype=np.uint8)
    archive = to_device(padded)
    producer = to_device(np.array([0, 0, len(file) & 0xffffffff, len(file) >> 32], np.uint32))
    src = CompressedInput()
    src.bytes = ConstBytes(archive.data_ptr(), archive.numel())
    src.encoder_result = producer.data_ptr()
    src.trusted_image = api.image_spec(1, 300, 100)
    src.trusted_tile = TileShape()
    out = device_bytes(300 * 100 * 2)
    item = BatchItem()
    item.compressed_input = src
    item.output = api.view(out, 1, 300, 100, 600, out.numel())
    run = Run(cuda.Operation.decompress, [item], keep=[archive, producer, out])
    assert run.status == Status.success
    assert run.execute(cuda.decompress_async) == Status.success
    assert run.records()[0] == (5, 0, 0)


def test_trusted_producer_error_propagates(cuda_ready):
    archive = device_bytes(20000, fill=0)
    producer = to_device(np.array([5, 0, 0, 0], np.uint32))  # malformed_data from the producer
    src = CompressedInput()
    src.bytes = ConstBytes(archive.data_ptr(), archive.numel())
    src.encoder_result = producer.data_ptr()
    src.trusted_image = api.image_spec(1, 100, 40)
    src.trusted_tile = TileShape()
    out = device_bytes(100 * 40 * 2)
    item = BatchItem()
    item.compressed_input = src
    item.output = api.view(out, 1, 100, 40, 200, out.numel())
    run = Run(cuda.Operation.decompress, [item], keep=[archive, producer, out])
    assert run.status == Status.success
    assert run.execute(cuda.decompress_async) == Status.success
    assert run.records()[0] == (5, 0, 0)
    assert np.all(host(out) == SENTINEL)  # nothing consumed
