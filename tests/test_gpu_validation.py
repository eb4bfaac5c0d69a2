"""Error behaviour of plan preparation and execution through the C ABI: the same requests the
reference's validation tests make, with the same statuses, and a failed preparation leaves the
caller's previous plan in place (reference tests/cuda_decoder_test.cpp:454-650,
tests/cuda_encoder_test.cpp:227-372, tests/cuda_calibration_test.cpp:408-600)."""
import ctypes as C

import numpy as np
import pytest

from support import SENTINEL, device_bytes, host, to_device
from tilestream_b200 import _native as N
from tilestream_b200 import api, cuda, workloads
from tilestream_b200.api import (BatchItem, ConstBytes, MutableBytes,
                                 ResultBuffer, Roi, Status, TileMapping, TileShape)

pytestmark = pytest.mark.gpu


class Handle:
    """A raw plan handle for the executors (the test owns and frees it)."""

    def __init__(self, value):
        self.handle = value


def cpp_item():
    """A BatchItem with the reference's C++ member defaults (C records start zeroed): pixel
    type uint16 in every image spec, tile 128x32 for trusted sources, gain 1.0."""
    item = BatchItem()
    for view in (item.input, item.output, item.compressed_input.trusted_image,
                 item.calibration.offset.map, item.calibration.gain.map):
        spec = view if isinstance(view, api.ImageSpec) else view.image
        spec.type = int(api.PixelType.uint16)
    item.compressed_input.trusted_tile = TileShape()
    item.calibration.gain.scalar = 1.0
    return item


def prepare(op, items, tile=None, previous=None):
    """ts_prepare_batch with *plan preset to `previous`: (status, handle after the call)."""
    items = list(items)
    arr = (BatchItem * max(1, len(items)))(*items)
    req = api.BatchRequest(int(op), C.cast(arr, C.POINTER(BatchItem)) if items else None,
                           len(items), tile if tile is not None else TileShape())
    h = C.c_void_p(previous)
    st = Status(N.lib().ts_prepare_batch(C.byref(req), C.byref(h), None))
    return st, h.value


def destroy(handle):
    if handle:
        N.lib().ts_plan_destroy(handle)


def workspace_for(handle):
    spec = api.WorkspaceSpec()
    N.lib().ts_plan_workspace_spec(handle, C.byref(spec))
    st, n = api.workspace_size(spec)
    assert st == Status.success
    return n


def pageable_access() -> bool:
    import torch
    torch.cuda.init()
    rt = C.CDLL("libcudart.so.12")
    v = C.c_int(0)
    assert rt.cudaDeviceGetAttribute(C.byref(v), 88, 0) == 0  # PageableMemoryAccess
    return v.value != 0


# ---- decoder --------------------------------------------------------------------------------

class Dec:
    """A 200x70 uint16 archive (128x32 tiles: 2 x 3 tiles) decoded whole as an ROI."""

    def __init__(self, o):
        # A smooth noisy field (no constant tiles, so tile 0 is predictive).
        rng = np.random.default_rng(23)
        y, x = np.mgrid[0:70, 0:200]
        self.frame = (1000 + 3 * x + 2 * y + rng.integers(0, 8, (70, 200))).astype(np.uint16)
        self.file = o.compress_image(self.frame, (128, 32))
        st, self.meta = api.parse_metadata(self.file)
        assert st == Status.success
        self.bytes = to_device(np.frombuffer(self.file, np.uint8))
        self.out = device_bytes(200 * 70 * 2)
        self.item = cpp_item()
        src = self.item.compressed_input
        src.bytes = ConstBytes(self.bytes.data_ptr(), len(self.file))
        src.metadata = self.meta.handle
        self.item.output = api.view(self.out, 1, 200, 70, 400, 200 * 70 * 2)
        self.item.roi = Roi(0, 0, 200, 70)

    def copy(self):
        c = BatchItem()
        C.pointer(c)[0] = self.item
        return c


@pytest.fixture(scope="module")
def dec(oracle_lib):
    return Dec(oracle_lib)


def test_empty_batches_are_no_ops(cuda_ready):
    for op, run in ((cuda.Operation.decompress, cuda.decompress_async),
                    (cuda.Operation.decode_roi, cuda.decode_roi_async),
                    (cuda.Operation.compress, cuda.compress_async),
                    (cuda.Operation.calibrate, cuda.calibrate_async),
                    (cuda.Operation.decode_calibrate, cuda.decode_calibrate_async)):
        st, h = prepare(op, [])
        assert st == Status.success
        assert workspace_for(h) == 0
        assert run(Handle(h), MutableBytes(None, 0), ResultBuffer(None, 0)) == Status.success
        if op != cuda.Operation.compress:
            assert cuda.compress_async(Handle(h), MutableBytes(None, 0),
                                       ResultBuffer(None, 0)) == Status.invalid_argument
        destroy(h)


def test_decoder_rejects_invalid_regions_and_views(cuda_ready, dec):
    st, previous = prepare(cuda.Operation.decode_roi, [dec.item])
    assert st == Status.success

    def attempt(item, status, op=cuda.Operation.decode_roi):
        got, h = prepare(op, [item], previous=previous)
        assert got == status, (got, status)
        assert h == previous

    for roi in ((0, 0, 0, 70), (0, 0, 200, 0), (1, 0, 200, 70), (0, 70, 200, 1), (200, 0, 1, 1),
                (0xFFFFFFFF, 0, 2, 1), (0, 0xFFFFFFFF, 1, 2)):
        c = dec.copy()
        c.roi = Roi(*roi)
        w, h = max(roi[2], 1), max(roi[3], 1)
        c.output = api.view(dec.out, 1, w, h, w * 2, 200 * 70 * 2)
        attempt(c, Status.invalid_roi)
    c = dec.copy()
    c.roi = Roi(10, 10, 20, 20)
    attempt(c, Status.invalid_argument)  # output shape is not the region's
    c.output = api.view(dec.out, 1, 20, 20, 40, 200 * 70 * 2)
    st, h = prepare(cuda.Operation.decode_roi, [c], previous=previous)
    assert st == Status.success and h != previous
    previous = h
    c.output = api.view(dec.out, 2, 20, 20, 80, 200 * 70 * 2)
    attempt(c, Status.invalid_argument)  # output type is not the archive's
    c = dec.copy()
    c.output.capacity_bytes = 100
    attempt(c, Status.buffer_too_small)
    c = dec.copy()
    c.output.data = dec.out.data_ptr() + 1
    attempt(c, Status.invalid_argument)  # misaligned output
    c = dec.copy()
    c.output.data = dec.bytes.data_ptr()
    attempt(c, Status.invalid_argument)  # output overlaps the archive
    c = dec.copy()
    c.output = api.view(dec.out, 1, 199, 70, 398, 200 * 70 * 2)
    attempt(c, Status.invalid_argument, cuda.Operation.decompress)
    destroy(previous)


def test_decoder_rejects_inconsistent_sources(cuda_ready, dec):
    st, base = prepare(cuda.Operation.decode_roi, [dec.item])
    assert st == Status.success

    def expect(item, status):
        got, h = prepare(cuda.Operation.decode_roi, [item], previous=base)
        assert got == status, (got, status)
        if got != Status.success:
            assert h == base
        return h

    c = dec.copy()
    c.compressed_input.bytes.size = len(dec.file) - 1
    expect(c, Status.buffer_too_small)
    c = dec.copy()
    c.compressed_input.bytes.data = dec.bytes.data_ptr() + 2
    expect(c, Status.invalid_argument)
    c = dec.copy()
    c.compressed_input.metadata = None
    expect(c, Status.invalid_argument)
    c = dec.copy()
    c.compressed_input.encoder_result = dec.out.data_ptr()
    expect(c, Status.invalid_argument)  # metadata and an encoder result together

    # Mappings list exactly the intersecting tiles (1 and 3), aligned, without overlap.
    tiles = dec.meta.tiles
    c = dec.copy()
    c.roi = Roi(130, 0, 10, 40)
    c.output = api.view(dec.out, 1, 10, 40, 20, 200 * 70 * 2)
    good = (TileMapping * 2)(TileMapping(1, int(tiles[1]["offset"])),
                             TileMapping(3, int(tiles[3]["offset"])))
    c.compressed_input.mappings = good
    c.compressed_input.mapping_count = 2
    base = expect(c, Status.success)
    for bad in ([(1, int(tiles[1]["offset"]))], [(3, 0), (1, 0)], [(1, 2), (3, 1024)],
                [(1, 0), (3, 4)], [(1, 0), (3, len(dec.file))]):
        arr = (TileMapping * len(bad))(*[TileMapping(t, o) for t, o in bad])
        c.compressed_input.mappings = arr
        c.compressed_input.mapping_count = len(bad)
        expect(c, Status.invalid_argument)
    c.compressed_input.mappings = None
    expect(c, Status.invalid_argument)

    # Fabricated metadata that would send device reads outside a payload.
    t0 = tiles.copy()
    assert int(t0[0]["mode"]) == int(api.TileMode.predict_bitpack)
    segs = dec.meta.segments
    for mutation in range(5):
        t, s = tiles.copy(), segs.copy()
        if mutation == 0:
            t[0]["length"] = 1 << 16
        elif mutation == 1:
            t[0]["first_segment"] = len(s)
        elif mutation == 2:
            s[3]["payload_bytes"] += 4
        elif mutation == 3:
            s[0]["bit_width"] = 17
        else:
            t = t[:-1]
        st, fabricated = api.ImageMetadata.create(dec.meta.image, dec.meta.tile,
                                                  dec.meta.file_bytes, t, s)
        assert st == Status.success
        c = dec.copy()
        c.compressed_input.metadata = fabricated.handle
        expect(c, Status.malformed_data)

    # Two items writing the same output; then a uint16 and a float32 item in one batch.
    pair = [dec.copy(), dec.copy()]
    assert prepare(cuda.Operation.decode_roi, pair)[0] == Status.invalid_argument
    second = device_bytes(200 * 70 * 2)
    pair[1].output.data = second.data_ptr()
    st, h = prepare(cuda.Operation.decode_roi, pair)
    assert st == Status.success
    destroy(h)
    floats = workloads.field_frame(5, 5, seed=1)
    import oracle
    ffile = oracle.Oracle().compress_image(floats)
    st, fmeta = api.parse_metadata(ffile)
    fdev = to_device(np.frombuffer(ffile, np.uint8))
    fsrc = cpp_item().compressed_input
    fsrc.bytes = ConstBytes(fdev.data_ptr(), len(ffile))
    fsrc.metadata = fmeta.handle
    pair[1].compressed_input = fsrc
    pair[1].output = api.view(second, 2, 5, 5, 20, 100)
    pair[1].roi = Roi(0, 0, 5, 5)
    assert prepare(cuda.Operation.decode_roi, pair)[0] == Status.invalid_argument
    destroy(base)


def test_trusted_sources_need_complete_shapes(cuda_ready, dec):
    encoded = device_bytes(len(dec.file))
    result = device_bytes(16, fill=0)
    c = dec.copy()
    c.compressed_input = cpp_item().compressed_input
    c.compressed_input.bytes = ConstBytes(encoded.data_ptr(), len(dec.file))
    c.compressed_input.encoder_result = result.data_ptr()
    c.compressed_input.trusted_image = api.image_spec(1, 200, 70)
    st, bound = api.compress_bound(api.image_spec(1, 200, 70), TileShape())
    assert prepare(cuda.Operation.decode_roi, [c])[0] == Status.buffer_too_small
    large = device_bytes(bound)
    c.compressed_input.bytes = ConstBytes(large.data_ptr(), bound)
    st, h = prepare(cuda.Operation.decode_roi, [c])
    assert st == Status.success
    destroy(h)
    c.compressed_input.trusted_tile = TileShape(16, 16)
    assert prepare(cuda.Operation.decode_roi, [c])[0] == Status.invalid_argument
    c.compressed_input.trusted_tile = TileShape()
    c.compressed_input.trusted_image = api.ImageSpec(5, 200, 70)
    assert prepare(cuda.Operation.decode_roi, [c])[0] == Status.unsupported_type
    c.compressed_input.trusted_image = api.image_spec(1, 200, 70)
    c.compressed_input.encoder_result = result.data_ptr() + 4
    assert prepare(cuda.Operation.decode_roi, [c])[0] == Status.invalid_argument
    c.compressed_input.encoder_result = result.data_ptr()
    c.compressed_input.metadata = dec.meta.handle
    assert prepare(cuda.Operation.decode_roi, [c])[0] == Status.invalid_argument
    # The consuming result buffer must not alias the producer's result.
    c.compressed_input.metadata = None
    st, h = prepare(cuda.Operation.decode_roi, [c])
    assert st == Status.success
    ws = device_bytes(max(workspace_for(h), 1))
    assert cuda.decode_roi_async(Handle(h), MutableBytes(ws.data_ptr(), ws.numel()),
                                 ResultBuffer(result.data_ptr(), 1)) == Status.invalid_argument
    destroy(h)


# ---- encoder --------------------------------------------------------------------------------

class Enc:
    def __init__(self):
        rng = np.random.default_rng(3)
        self.frame = rng.integers(0, 65536, (33, 129), dtype=np.uint16)
        self.input = to_device(self.frame)
        st, self.bound = api.compress_bound(api.image_spec(1, 129, 33), TileShape())
        self.output = device_bytes(self.bound + 64)
        self.item = cpp_item()
        self.item.input = api.const_view(self.input, 1, 129, 33, 258, self.input.numel())
        self.item.compressed_output = MutableBytes(self.output.data_ptr(), self.bound)

    def copy(self):
        c = BatchItem()
        C.pointer(c)[0] = self.item
        return c


def test_encoder_rejects_invalid_requests_and_keeps_previous_plan(cuda_ready):
    e = Enc()
    st, previous = prepare(cuda.Operation.compress, [e.item])
    assert st == Status.success

    def attempt(item, status, count=None):
        got, h = prepare(cuda.Operation.compress, [item], previous=previous)
        assert got == status, (got, status)
        assert h == previous

    c = e.copy()
    c.input.image.type = 9
    attempt(c, Status.unsupported_type)
    c = e.copy()
    c.input.image.width = 0
    attempt(c, Status.invalid_argument)
    c = e.copy()
    c.input.pitch_bytes = 2
    attempt(c, Status.invalid_argument)
    c = e.copy()
    c.input.data = e.input.data_ptr() + 1
    attempt(c, Status.invalid_argument)
    c = e.copy()
    c.input.capacity_bytes = 10
    attempt(c, Status.buffer_too_small)
    c = e.copy()
    c.compressed_output = MutableBytes(None, e.bound)
    attempt(c, Status.invalid_argument)
    c = e.copy()
    c.compressed_output = MutableBytes(e.output.data_ptr() + 2, e.bound)
    attempt(c, Status.invalid_argument)
    c = e.copy()
    c.compressed_output.size = e.bound - 1
    attempt(c, Status.buffer_too_small)
    c = e.copy()
    c.compressed_output.size = (1 << 64) - 1
    attempt(c, Status.size_overflow)
    c = e.copy()
    c.compressed_output = MutableBytes(e.input.data_ptr(), e.bound)
    attempt(c, Status.invalid_argument)  # output overlaps the input
    if not pageable_access():
        host_buf = np.zeros(e.bound + 16, np.uint8)
        aligned = (host_buf.ctypes.data + 3) // 4 * 4
        c = e.copy()
        c.compressed_output = MutableBytes(aligned, e.bound)
        attempt(c, Status.invalid_argument)  # host memory the device cannot reach

    second = device_bytes(e.bound)
    pair = [e.copy(), e.copy()]
    assert prepare(cuda.Operation.compress, pair, previous=previous) == \
        (Status.invalid_argument, previous)  # two items, one output
    pair[1].compressed_output = MutableBytes(second.data_ptr(), e.bound)
    pair[1].input.image.type = 2
    pair[1].input.pitch_bytes = 129 * 4
    pair[1].input.image.height = 1
    assert prepare(cuda.Operation.compress, pair, previous=previous) == \
        (Status.invalid_argument, previous)  # mixed pixel types
    assert prepare(cuda.Operation.compress, [e.item], TileShape(32, 128), previous) == \
        (Status.invalid_argument, previous)
    assert prepare(cuda.Operation.calibrate, [e.item], previous=previous) == \
        (Status.invalid_argument, previous)
    req = api.BatchRequest(int(cuda.Operation.compress), None, 1, TileShape())
    h = C.c_void_p(previous)
    assert N.lib().ts_prepare_batch(C.byref(req), C.byref(h), None) == Status.invalid_argument
    arr = (BatchItem * 1)(e.item)
    req = api.BatchRequest(int(cuda.Operation.compress), C.cast(arr, C.POINTER(BatchItem)),
                           (1 << 32), TileShape())
    assert N.lib().ts_prepare_batch(C.byref(req), C.byref(h), None) == Status.resource_limit
    assert h.value == previous
    # Inputs are read-only and may be shared.
    pair = [e.copy(), e.copy()]
    pair[1].compressed_output = MutableBytes(second.data_ptr(), e.bound)
    st, h2 = prepare(cuda.Operation.compress, pair)
    assert st == Status.success
    destroy(h2)
    destroy(previous)


def test_encoder_rejected_executions_leave_buffers_untouched(cuda_ready, oracle_lib):
    import torch
    e = Enc()
    st, h = prepare(cuda.Operation.compress, [e.item])
    assert st == Status.success
    n = workspace_for(h)
    ws = device_bytes(n)
    large = device_bytes(n + 1024)
    results = device_bytes(4 * 16)
    rec = results.data_ptr()
    plan = Handle(h)

    def attempt(scratch, buf, status):
        assert cuda.compress_async(plan, scratch, buf) == status

    attempt(MutableBytes(ws.data_ptr(), n - 1), ResultBuffer(rec, 1), Status.buffer_too_small)
    attempt(MutableBytes(None, 0), ResultBuffer(rec, 1), Status.buffer_too_small)
    attempt(MutableBytes(large.data_ptr() + 128, n), ResultBuffer(rec, 1),
            Status.invalid_argument)  # workspace not aligned to 256 bytes
    full = MutableBytes(ws.data_ptr(), n)
    attempt(full, ResultBuffer(rec, 0), Status.buffer_too_small)
    attempt(full, ResultBuffer(None, 1), Status.invalid_argument)
    attempt(full, ResultBuffer(rec + 4, 1), Status.invalid_argument)
    attempt(full, ResultBuffer(rec, ((1 << 64) - 1) // 8), Status.size_overflow)
    attempt(MutableBytes(e.output.data_ptr(), n), ResultBuffer(rec, 1), Status.invalid_argument)
    attempt(full, ResultBuffer(e.output.data_ptr(), 1), Status.invalid_argument)
    attempt(full, ResultBuffer(e.input.data_ptr(), 1), Status.invalid_argument)
    attempt(full, ResultBuffer(ws.data_ptr(), 1), Status.invalid_argument)
    torch.cuda.synchronize()
    assert np.all(host(e.output) == SENTINEL)
    assert np.all(host(results) == SENTINEL)
    assert cuda.compress_async(plan, full, ResultBuffer(rec, 1)) == Status.success
    torch.cuda.synchronize()
    r = host(results)[:16].view(np.uint64)
    assert int(r[0]) == 0
    got = host(e.output)[:int(r[1])].tobytes()
    assert got == oracle_lib.compress_image(e.frame)
    destroy(h)


# ---- calibration ----------------------------------------------------------------------------

class Cal:
    """A 64x40 uint16 image calibrated to FP32 with an offset map; a fused ROI item too."""

    def __init__(self, o):
        rng = np.random.default_rng(14)
        self.image = rng.integers(0, 1 << 12, (40, 64), dtype=np.uint16)
        self.input = to_device(self.image)
        self.out = device_bytes(64 * 40 * 4)
        self.omap = to_device(rng.uniform(0, 10, (40, 64)).astype(np.float32))
        self.item = cpp_item()
        self.item.input = api.const_view(self.input, 1, 64, 40, 128, self.input.numel())
        self.item.output = api.view(self.out, 2, 64, 40, 256, self.out.numel())
        self.item.calibration.offset.kind = cuda.ParameterKind.map
        self.item.calibration.offset.map = api.const_view(self.omap, 2, 64, 40, 256,
                                                          self.omap.numel())
        self.item.calibration.gain.scalar = 1.0
        self.file = o.compress_image(self.image)
        st, self.meta = api.parse_metadata(self.file)
        self.src = to_device(np.frombuffer(self.file, np.uint8))
        self.roi_out = device_bytes(30 * 20 * 4)
        self.roi_map = to_device(rng.uniform(0, 10, (20, 30)).astype(np.float32))
        self.fused = cpp_item()
        self.fused.compressed_input.bytes = ConstBytes(self.src.data_ptr(), len(self.file))
        self.fused.compressed_input.metadata = self.meta.handle
        self.fused.roi = Roi(5, 6, 30, 20)
        self.fused.output = api.view(self.roi_out, 2, 30, 20, 120, self.roi_out.numel())
        self.fused.calibration.offset.kind = cuda.ParameterKind.map
        self.fused.calibration.offset.map = api.const_view(self.roi_map, 2, 30, 20, 120,
                                                           self.roi_map.numel())
        self.fused.calibration.gain.scalar = 1.0

    @staticmethod
    def copy(item):
        c = BatchItem()
        C.pointer(c)[0] = item
        return c


def attempt_cal(op, item, status):
    st, h = prepare(op, [item])
    assert st == status, (st, status)
    assert (h is None) == (status != Status.success)
    destroy(h)


def test_calibration_rejects_invalid_outputs_and_maps(cuda_ready, oracle_lib):
    k = Cal(oracle_lib)
    op = cuda.Operation.calibrate
    attempt_cal(op, k.item, Status.success)
    c = k.copy(k.item)
    c.output.image.type = 1
    attempt_cal(op, c, Status.invalid_argument)
    c = k.copy(k.item)
    c.output.image.width = 63
    attempt_cal(op, c, Status.invalid_argument)
    c = k.copy(k.item)
    c.output.data = None
    attempt_cal(op, c, Status.invalid_argument)
    for field, value, status in (("width", 63, Status.invalid_argument),
                                 ("type", 1, Status.invalid_argument),
                                 ("type", 7, Status.unsupported_type)):
        c = k.copy(k.item)
        setattr(c.calibration.offset.map.image, field, value)
        attempt_cal(op, c, status)
    for pitch in (64 * 4 - 4, 64 * 4 + 2):
        c = k.copy(k.item)
        c.calibration.offset.map.pitch_bytes = pitch
        attempt_cal(op, c, Status.invalid_argument)
    c = k.copy(k.item)
    c.calibration.offset.map.capacity_bytes = 64 * 4 * 39
    attempt_cal(op, c, Status.buffer_too_small)
    c = k.copy(k.item)
    c.calibration.offset.map.data = None
    attempt_cal(op, c, Status.invalid_argument)
    c = k.copy(k.item)
    c.calibration.gain.kind = 5
    attempt_cal(op, c, Status.invalid_argument)
    c = k.copy(k.item)
    c.calibration.gain.kind = cuda.ParameterKind.map  # a map kind without a map
    attempt_cal(op, c, Status.invalid_argument)
    # Never in place, and outputs do not overlap maps.
    c = k.copy(k.item)
    c.output.data = k.omap.data_ptr()
    c.output.capacity_bytes = k.omap.numel()
    attempt_cal(op, c, Status.invalid_argument)
    if not pageable_access():
        hostmap = np.zeros((40, 64), np.float32)
        c = k.copy(k.item)
        c.calibration.offset.map.data = hostmap.ctypes.data
        c.calibration.offset.map.capacity_bytes = hostmap.nbytes
        attempt_cal(op, c, Status.invalid_argument)


def test_calibration_rejects_inconsistent_batches(cuda_ready, oracle_lib):
    k = Cal(oracle_lib)
    other = workloads.field_frame(64, 40, seed=15)
    other_in = to_device(other)
    other_out = device_bytes(64 * 40 * 4)
    pair = [k.copy(k.item), k.copy(k.item)]
    pair[1].input = api.const_view(other_in, 2, 64, 40, 256, other_in.numel())
    pair[1].output = api.view(other_out, 2, 64, 40, 256, other_out.numel())
    assert prepare(cuda.Operation.calibrate, pair)[0] == Status.invalid_argument  # mixed types
    pair[1] = k.copy(k.item)
    assert prepare(cuda.Operation.calibrate, pair)[0] == Status.invalid_argument  # same output
    c = k.copy(k.item)
    c.input = api.const_view(other_in, 2, 64, 40, 256, other_in.numel())
    c.output = api.view(other_in, 2, 64, 40, 256, other_in.numel())
    attempt_cal(cuda.Operation.calibrate, c, Status.invalid_argument)  # in place
    c.input.image.type = 9
    attempt_cal(cuda.Operation.calibrate, c, Status.unsupported_type)


def test_fused_regions_and_outputs(cuda_ready, oracle_lib):
    k = Cal(oracle_lib)
    op = cuda.Operation.decode_calibrate
    attempt_cal(op, k.fused, Status.success)
    c = k.copy(k.fused)
    c.roi = Roi(5, 6, 0, 20)
    attempt_cal(op, c, Status.invalid_roi)
    c.roi = Roi(40, 6, 30, 20)
    attempt_cal(op, c, Status.invalid_roi)
    c = k.copy(k.fused)
    c.output.image.type = 1
    attempt_cal(op, c, Status.invalid_argument)
    c = k.copy(k.fused)
    c.calibration.offset.map = k.item.calibration.offset.map  # maps follow the region
    attempt_cal(op, c, Status.invalid_argument)
    c = k.copy(k.fused)
    c.output = k.item.output
    c.calibration = cpp_item().calibration
    attempt_cal(op, c, Status.invalid_argument)


def test_execution_needs_matching_plan_and_workspace(cuda_ready, oracle_lib):
    import torch
    k = Cal(oracle_lib)
    st, standalone = prepare(cuda.Operation.calibrate, [k.item])
    assert st == Status.success
    st, combined = prepare(cuda.Operation.decode_calibrate, [k.fused])
    assert st == Status.success
    assert workspace_for(standalone) == 0
    results = device_bytes(16, fill=0xFF)
    rec = ResultBuffer(results.data_ptr(), 1)
    n = workspace_for(combined)
    ws = device_bytes(max(n, 1))
    full = MutableBytes(ws.data_ptr(), n)
    none = MutableBytes(None, 0)
    assert cuda.decode_calibrate_async(Handle(standalone), none, rec) == Status.invalid_argument
    assert cuda.calibrate_async(Handle(combined), full, rec) == Status.invalid_argument
    assert cuda.decode_roi_async(Handle(combined), full, rec) == Status.invalid_argument
    if n > 0:
        assert cuda.decode_calibrate_async(Handle(combined), MutableBytes(ws.data_ptr(), n - 1),
                                           rec) == Status.buffer_too_small
    assert cuda.calibrate_async(Handle(standalone), none, rec) == Status.success
    torch.cuda.synchronize()
    r = host(results).view(np.uint64)
    assert int(r[0]) == 0 and int(r[1]) == 64 * 40 * 4
    destroy(standalone)
    destroy(combined)
