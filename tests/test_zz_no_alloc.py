"""The allocation-free encode entry point (ts_compress_noalloc in include/tilestream_c.h).

It serves callers that cannot allocate device memory while they encode (GPU memory reserved in
full by another allocator, acquisition loops that must not stall on an allocator, deployments
without dynamic allocation after start-up). Its scratch is a fixed array in device memory shared
by every call, so these tests check that two calls in a row - the second reusing what the first
left in the array - each produce exactly the file of the plan-based compress_async path and of
the CPU oracle. The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from support import SENTINEL, Run, device_bytes, host, to_device
from tilestream_b200 import _native as N
from tilestream_b200 import api, cuda, workloads
from tilestream_b200.api import BatchItem, Status, TileShape

pytestmark = pytest.mark.gpu


def plan_encode(frame, ptype, tile):
    """The existing entry point: prepare_batch + compress_async, one image."""
    h, w = frame.shape
    dev = to_device(frame)
    st, bound = api.compress_bound(api.image_spec(ptype, w, h), TileShape(*tile))
    out = device_bytes(bound)
    item = BatchItem()
    item.input = api.const_view(dev, ptype, w, h, w * frame.itemsize, dev.numel())
    item.compressed_output = api.MutableBytes(out.data_ptr(), bound)
    run = Run(cuda.Operation.compress, [item], tile=TileShape(*tile), keep=[dev, out])
    assert run.status == Status.success
    assert run.execute(cuda.compress_async) == Status.success
    rec = run.records()[0]
    assert rec[0] == 0
    return host(out)[:rec[2]].tobytes(), rec


def noalloc_call(frame, ptype, tile, stream):
    """Enqueues one allocation-free encode; returns (status, device input, output, result)."""
    h, w = frame.shape
    dev = to_device(frame)
    st, bound = api.compress_bound(api.image_spec(ptype, w, h), TileShape(*tile))
    out = device_bytes(bound + 64)
    result = device_bytes(16, fill=0xFF)
    status = N.lib().ts_compress_noalloc(
        api.const_view(dev, ptype, w, h, w * frame.itemsize, dev.numel()), TileShape(*tile),
        api.MutableBytes(out.data_ptr(), bound), result.data_ptr(), stream.cuda_stream)
    return Status(status), dev, out, result, bound


def record(result):
    r = host(result).view(np.uint32)
    return int(r[0]), int(r[1]), int(r[2]) | (int(r[3]) << 32)


def test_two_calls_in_a_row_match_the_plan_path(cuda_ready, oracle_lib):
    torch = cuda_ready
    stream = torch.cuda.current_stream()
    first = workloads.detector_frame(1000, 700, seed=61)        # 8 x 22 tiles of 128x32
    second = workloads.field_frame(3000, 2000, seed=62)         # more tiles than the first
    calls = [(first, 1, (128, 32)), (second, 2, (64, 64))]
    pending = []
    for frame, ptype, tile in calls:
        st, dev, out, result, bound = noalloc_call(frame, ptype, tile, stream)
        assert st == Status.success, st
        pending.append((frame, ptype, tile, dev, out, result, bound))
    torch.cuda.synchronize()
    for frame, ptype, tile, dev, out, result, bound in pending:
        want, want_rec = plan_encode(frame, ptype, tile)
        got_rec = record(result)
        assert got_rec == want_rec
        data = host(out)
        assert data[:got_rec[2]].tobytes() == want
        assert want == oracle_lib.compress_image(frame, tile)
        assert np.all(data[bound:] == SENTINEL)
    # Again in the other order: the array now holds the larger image's flags.
    for frame, ptype, tile in reversed(calls):
        st, dev, out, result, bound = noalloc_call(frame, ptype, tile, stream)
        assert st == Status.success
        torch.cuda.synchronize()
        want, want_rec = plan_encode(frame, ptype, tile)
        assert record(result) == want_rec
        assert host(out)[:want_rec[2]].tobytes() == want


def test_rejects_images_beyond_the_scratch_limit(cuda_ready):
    torch = cuda_ready
    limit = N.lib().ts_compress_noalloc_max_tiles()
    assert limit == 131070
    # 128 x 1025 tiles of 128x32 (1 GiB of uint16): one more tile row than fits.
    w, h = 128 * 128, 32 * 1025
    assert (w // 128) * (h // 32) > limit
    dev = device_bytes(w * h * 2, fill=0)
    st, bound = api.compress_bound(api.image_spec(1, w, h), TileShape())
    out = device_bytes(bound)
    result = device_bytes(16, fill=0x33)
    status = N.lib().ts_compress_noalloc(api.const_view(dev, 1, w, h, w * 2, dev.numel()),
                                         TileShape(), api.MutableBytes(out.data_ptr(), bound),
                                         result.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert Status(status) == Status.resource_limit
    torch.cuda.synchronize()
    assert bool((out[:4096] == SENTINEL).all()) and bool((out[-4096:] == SENTINEL).all())
    assert np.all(host(result) == 0x33)
    del dev, out
