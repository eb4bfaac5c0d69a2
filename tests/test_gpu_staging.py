"""ROI staging on the GPU: the payloads of the tiles that intersect an ROI are copied from an
archive in pinned host memory, device memory or pageable host memory (one run per tile row: a
staging kernel for the first two, one copy per run for the last), on a copy stream; the ROI is
then decoded from the staged tiles on another stream. Decoded pixels must
equal the crop of the source frame (reference intersecting tiles, tests/cuda_decoder_test.cpp:
19-31; staged tiles, cuda_decoder_test.cpp:40-82)."""
import numpy as np
import pytest

import oracle
from support import device_bytes, host, torch
from tilestream_b200 import api, cuda, workloads
from tilestream_b200.api import (BatchItem, Calibration, CompressedInput, ConstBytes,
                                 MutableBytes, Roi, Status, TileMapping)

pytestmark = pytest.mark.gpu


def stage_and_decode(meta, archive_ptr, archive_len, roi, ptype, calibrated=False):
    """Stages `roi` on a copy stream, decodes it on the current stream after an event. Returns
    (record, output bytes, staging info)."""
    t = torch()
    st, need = cuda.roi_staging_size(meta, Roi(*roi))
    assert st == Status.success
    staging = device_bytes(need.bytes)
    maps = (TileMapping * need.tiles)()
    copy = t.cuda.Stream()
    st, info = cuda.stage_roi_tiles(meta, Roi(*roi), ConstBytes(archive_ptr, archive_len),
                                    MutableBytes(staging.data_ptr(), staging.numel()), maps,
                                    copy)
    assert st == Status.success, st
    staged = t.cuda.Event()
    staged.record(copy)
    compute = t.cuda.current_stream()
    compute.wait_event(staged)
    src = CompressedInput()
    src.bytes = ConstBytes(staging.data_ptr(), need.bytes)
    src.metadata = meta.handle
    src.mappings = maps
    src.mapping_count = need.tiles
    x, y, w, h = roi
    otype = api.PixelType.float32 if calibrated else ptype
    out = device_bytes(w * h * api.sample_bytes(otype))
    item = BatchItem()
    item.compressed_input = src
    item.output = api.view(out, otype, w, h, w * api.sample_bytes(otype), out.numel())
    item.roi = Roi(*roi)
    if calibrated:
        cal = Calibration()
        cal.offset.scalar = 100.0
        cal.gain.scalar = 1.05
        item.calibration = cal
    op = cuda.Operation.decode_calibrate if calibrated else cuda.Operation.decode_roi
    st, plan = cuda.prepare_batch(cuda.make_request(op, [item]), None, compute)
    assert st == Status.success, st
    ws = t.empty(max(plan.workspace_bytes(), 256), dtype=t.uint8, device="cuda")
    res = device_bytes(16, fill=0xFF)
    run = cuda.decode_calibrate_async if calibrated else cuda.decode_roi_async
    assert run(plan, MutableBytes(ws.data_ptr(), ws.numel()), res, compute) == Status.success
    t.cuda.synchronize()
    rec = host(res).view(np.uint64)
    return (int(rec[0]), int(rec[1])), host(out), info


def test_staged_rois_match_crop(cuda_ready, oracle_lib):
    t = torch()
    rng = np.random.default_rng(31)
    for ptype in (oracle.UINT16, oracle.FLOAT32):
        frame = (workloads.detector_frame(1000, 600, 41) if ptype == oracle.UINT16
                 else workloads.field_frame(1000, 600, 42))
        for tile in api.TILE_SHAPES:
            file = oracle_lib.compress_image(frame, tile)
            st, meta = api.parse_metadata(np.frombuffer(file, dtype=np.uint8))
            pageable = np.frombuffer(file, dtype=np.uint8).copy()
            pinned = t.from_numpy(pageable.copy()).pin_memory()
            on_device = pinned.to("cuda")
            sources = (pinned.data_ptr(), on_device.data_ptr(), pageable.ctypes.data)
            rois = [(0, 0, 1000, 600), (999, 599, 1, 1), (tile[0] - 3, tile[1] - 2, 7, 5)]
            for _ in range(4):
                x, y = int(rng.integers(0, 1000)), int(rng.integers(0, 600))
                rois.append((x, y, int(rng.integers(1, 1001 - x)), int(rng.integers(1, 601 - y))))
            for k, roi in enumerate(rois):
                rec, out, info = stage_and_decode(meta, sources[k % 3], len(file), roi,
                                                  api.PixelType(ptype))
                x, y, w, h = roi
                want = frame[y:y + h, x:x + w]
                assert rec == (0, want.nbytes)
                assert np.array_equal(out.view(frame.dtype).reshape(h, w), want)
                assert 1 <= info.copies <= (y + h - 1) // tile[1] - y // tile[1] + 1


def test_staged_calibrated_roi_equals_resident_decode(cuda_ready, oracle_lib):
    """decode_calibrate from staged tiles equals decode_calibrate from the whole archive on the
    device, bit for bit."""
    from support import gpu_decode
    t = torch()
    frame = workloads.detector_frame(2000, 1200, seed=43)
    file = oracle_lib.compress_image(frame, (64, 64))
    st, meta = api.parse_metadata(np.frombuffer(file, dtype=np.uint8))
    pinned = t.from_numpy(np.frombuffer(file, dtype=np.uint8).copy()).pin_memory()
    roi = (130, 70, 1500, 900)
    rec, out, _ = stage_and_decode(meta, pinned.data_ptr(), len(file), roi,
                                   api.PixelType.uint16, calibrated=True)
    cal = Calibration()
    cal.offset.scalar = 100.0
    cal.gain.scalar = 1.05
    st, rec2, out2, _ = gpu_decode(file, roi=roi, operation=cuda.Operation.decode_calibrate,
                                   calibration=cal)
    assert st == Status.success and rec2[0] == 0
    assert rec == (0, roi[2] * roi[3] * 4) and rec2[2] == roi[2] * roi[3] * 4
    assert np.array_equal(out[:roi[2] * roi[3] * 4], out2[:roi[2] * roi[3] * 4])


def test_out_of_order_payloads(cuda_ready, oracle_lib):
    """Metadata whose tiles are stored out of file order: each tile is its own run, and the
    staged ROI still decodes to the crop."""
    from test_staging import permuted_archive
    t = torch()
    frame = workloads.detector_frame(900, 500, seed=8)
    for tile in api.TILE_SHAPES:
        file, meta = permuted_archive(oracle_lib, frame, tile, seed=tile[1])
        pinned = t.from_numpy(np.frombuffer(file, dtype=np.uint8).copy()).pin_memory()
        for roi in ((0, 0, 900, 500), (100, 40, 333, 210)):
            rec, out, info = stage_and_decode(meta, pinned.data_ptr(), len(file), roi,
                                              api.PixelType.uint16)
            x, y, w, h = roi
            want = frame[y:y + h, x:x + w]
            assert rec == (0, want.nbytes)
            assert np.array_equal(out.view(np.uint16).reshape(h, w), want)


def test_staged_rois_as_one_mixed_batch(cuda_ready, oracle_lib):
    """Several ROIs of uint16 and FP32 archives staged from pinned memory, then decoded as one
    mixed batch (decode_roi and decode_calibrate items with their tile mappings): every output
    equals the crop (or its calibrated form) of the source frame."""
    t = torch()
    rng = np.random.default_rng(37)
    copy = t.cuda.Stream()
    compute = t.cuda.current_stream()
    items, keep, checks = [], [], []
    for k, (ptype, tile) in enumerate([(oracle.UINT16, (128, 32)), (oracle.FLOAT32, (64, 64)),
                                       (oracle.UINT16, (256, 16))]):
        frame = (workloads.detector_frame(900, 500, 60 + k) if ptype == oracle.UINT16
                 else workloads.field_frame(900, 500, 60 + k))
        file = oracle_lib.compress_image(frame, tile)
        st, meta = api.parse_metadata(np.frombuffer(file, dtype=np.uint8))
        pinned = t.from_numpy(np.frombuffer(file, dtype=np.uint8).copy()).pin_memory()
        keep += [meta, pinned]
        for j in range(4):
            x, y = int(rng.integers(0, 900)), int(rng.integers(0, 500))
            roi = (x, y, int(rng.integers(1, 901 - x)), int(rng.integers(1, 501 - y)))
            st, need = cuda.roi_staging_size(meta, Roi(*roi))
            assert st == Status.success
            staging = device_bytes(need.bytes)
            maps = (TileMapping * need.tiles)()
            st, _ = cuda.stage_roi_tiles(meta, Roi(*roi), ConstBytes(pinned.data_ptr(), len(file)),
                                         MutableBytes(staging.data_ptr(), staging.numel()), maps,
                                         copy)
            assert st == Status.success, st
            calibrated = j % 2 == 1
            src = CompressedInput()
            src.bytes = ConstBytes(staging.data_ptr(), need.bytes)
            src.metadata = meta.handle
            src.mappings = maps
            src.mapping_count = need.tiles
            x, y, w, h = roi
            otype = api.PixelType.float32 if calibrated else api.PixelType(ptype)
            s = api.sample_bytes(otype)
            out = device_bytes(w * h * s)
            item = BatchItem()
            item.compressed_input = src
            item.output = api.view(out, otype, w, h, w * s, out.numel())
            item.roi = Roi(*roi)
            if calibrated:
                item.calibration = Calibration()
                item.calibration.offset.scalar = 100.0
                item.calibration.gain.scalar = 1.05
            op = cuda.Operation.decode_calibrate if calibrated else cuda.Operation.decode_roi
            items.append((op, item))
            keep += [staging, maps, out]
            region = np.ascontiguousarray(frame[y:y + h, x:x + w])
            want = (oracle_lib.calibrate_image(region, 100.0, 1.05) if calibrated else region)
            checks.append((out, want))
    staged = t.cuda.Event()
    staged.record(copy)
    compute.wait_event(staged)
    results = device_bytes(16 * len(items), fill=0xFF)
    st, batch = cuda.prepare_mixed_batch(items, results, compute, graph=False)
    assert st == Status.success, st
    assert batch.run(compute) == Status.success
    t.cuda.synchronize()
    recs = host(results).view(np.uint64).reshape(-1, 2)
    for k, (out, want) in enumerate(checks):
        assert int(recs[k, 0]) == 0 and int(recs[k, 1]) == want.nbytes, k
        got = host(out)[:want.nbytes].view(want.dtype).reshape(want.shape)
        assert np.array_equal(got.view(np.uint8), want.view(np.uint8)) or (
            want.dtype == np.float32 and np.all((got.view(np.uint32) == want.view(np.uint32)) |
                                                (np.isnan(got) & np.isnan(want)))), k
