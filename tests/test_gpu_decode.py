"""GPU decoder parity: every decoded word must equal the oracle's (the reference CPU codec's
algorithm), including signed zeros, infinities, NaN payloads, subnormals, partial and pitched
tiles, ROIs, staged tile subsets; pitch padding and everything outside the ROI stay untouched.
Modelled on the reference's tests/cuda_decoder_test.cpp."""
import json
import os

import numpy as np
import pytest

import oracle
from support import (SENTINEL, Run, crop, decode_item, device_bytes, gpu_decode, host, logical,
                     padding_untouched, parsed_source, to_device)
from tilestream_b200 import api, cuda, workloads
from tilestream_b200.api import CompressedInput, ConstBytes, Status, TileMapping

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def read_hex(name):
    with open(os.path.join(GOLDEN, name + ".hex")) as f:
        return bytes(int(t, 16) for t in f.read().split())


def test_golden_files_decode(cuda_ready):
    cases = json.load(open(os.path.join(GOLDEN, "cases.json")))
    for name, c in cases.items():
        file = read_hex(name)
        dtype = np.uint16 if c["type"] == 1 else np.uint32
        expected = np.array(c["pixels"], dtype=dtype).view(np.uint8)
        st, rec, out, pitch = gpu_decode(file)
        assert st == Status.success and rec == (0, 0, expected.size), name
        assert np.array_equal(out[:expected.size], expected), name


def _case_archive(o, c):
    return o.compress(c["bytes"], c["type"], c["width"], c["height"], c["pitch"], c["tile"])


@pytest.mark.parametrize("first", [13000000, 13000400])
def test_robustness_cases_whole_and_roi(cuda_ready, oracle_lib, first):
    """Seeded cases of the reference robustness suite: full decode into a padded pitch, and the
    case's ROI; both compared with the source pixels."""
    o = oracle_lib
    for seed in range(first, first + 200):
        c = o.case(seed)
        s = oracle.SAMPLE[c["type"]]
        w, h = c["width"], c["height"]
        file = _case_archive(o, c)
        src_px = logical(c["bytes"], w, h, c["pitch"], s)
        pitch = w * s + 2 * s
        st, rec, out, _ = gpu_decode(file, pitch=pitch)
        assert st == Status.success and rec == (0, 0, w * h * s), seed
        assert np.array_equal(logical(out, w, h, pitch, s), src_px), seed
        assert padding_untouched(out, w, h, pitch, s), seed
        roi = c["roi"]
        st, rec, out, rp = gpu_decode(file, roi=roi)
        assert st == Status.success and rec == (0, 0, roi[2] * roi[3] * s), seed
        want = crop(c["bytes"], c["pitch"], s, roi)
        assert np.array_equal(out[:want.size], want), seed


def test_batched_cases_one_plan(cuda_ready, oracle_lib):
    """Many uneven images of one pixel type and mixed tile geometries in one plan."""
    o = oracle_lib
    for parity in (0, 1):
        seeds = [13001000 + 2 * k + parity for k in range(120)]
        items, keep, expect = [], [], []
        for seed in seeds:
            c = o.case(seed)
            s = oracle.SAMPLE[c["type"]]
            file = _case_archive(o, c)
            src, meta, dev = parsed_source(file)
            pitch = c["width"] * s
            out = device_bytes(pitch * c["height"])
            items.append(decode_item(src, c["type"], out, c["width"], c["height"], pitch))
            keep += [meta, dev, out]
            expect.append((out, logical(c["bytes"], c["width"], c["height"], c["pitch"], s)))
        run = Run(cuda.Operation.decompress, items, keep=keep)
        assert run.status == Status.success
        assert run.execute(cuda.decompress_async) == Status.success
        recs = run.records()
        for (out, want), rec in zip(expect, recs):
            assert rec == (0, 0, want.size)
            assert np.array_equal(host(out)[:want.size], want)


@pytest.mark.parametrize("width", [1, 2, 31, 32, 33, 63, 64, 65, 127, 128, 129, 255, 256, 300])
def test_every_residual_width(cuda_ready, oracle_lib, width):
    """Rows built with every residual width 0..16 (uint16) and 0..32 (float32)."""
    rng = np.random.default_rng(width)
    for ptype, top in ((oracle.UINT16, 16), (oracle.FLOAT32, 32)):
        rows = []
        for bits in range(top + 1):
            mask = (1 << bits) - 1
            z = rng.integers(0, 1 << 32, width, dtype=np.uint64) & mask
            if width > 1:
                z[1] = mask  # force the full width
            if ptype == oracle.UINT16:
                d = np.where(z % 2 == 0, z // 2, -(z // 2).astype(np.int64) - 1)
                row = (np.cumsum(d.astype(np.int64)) + 400) % 65536
                rows.append(row.astype(np.uint16))
            else:
                acc = np.bitwise_xor.accumulate(z.astype(np.uint32))
                rows.append(acc.astype(np.uint32))
        img = np.stack(rows)
        for tile in api.TILE_SHAPES:
            file = o_compress(oracle_lib, img, tile)
            st, rec, out, pitch = gpu_decode(file)
            assert st == Status.success
            assert np.array_equal(out[:img.nbytes], img.view(np.uint8).reshape(-1)), (ptype, tile)


def o_compress(o, img, tile):
    return o.compress_image(img, tile)


def test_special_words_and_every_uint16(cuda_ready, oracle_lib):
    words = np.array([0x00000000, 0x80000000, 0x00000001, 0x807fffff, 0x00800000, 0x7f7fffff,
                      0xff800000, 0x7f800000, 0x7fc00000, 0xffc12345, 0x7f800001, 0x3f800000,
                      0x7fbfffff, 0xffffffff], dtype=np.uint32)
    rng = np.random.default_rng(7)
    img = rng.choice(words, size=(70, 300)).astype(np.uint32)
    for tile in api.TILE_SHAPES:
        file = oracle_lib.compress_image(img, tile)
        st, rec, out, _ = gpu_decode(file)
        assert st == Status.success and np.array_equal(out[:img.nbytes].view(np.uint32),
                                                       img.reshape(-1))
    every = np.arange(65536, dtype=np.uint16).reshape(256, 256)
    for img in (every, every[:, ::-1].copy(), every.T.copy()):
        for tile in api.TILE_SHAPES:
            file = oracle_lib.compress_image(img, tile)
            st, rec, out, _ = gpu_decode(file)
            assert st == Status.success and np.array_equal(out[:img.nbytes].view(np.uint16),
                                                           img.reshape(-1))


@pytest.mark.parametrize("tile", api.TILE_SHAPES)
def test_detector_frame_full_size(cuda_ready, oracle_lib, tile):
    """The 4096x4096 uint16 frame of the plain-GPU config, seed 2, for each tile shape."""
    frame = workloads.detector_frame(4096, 4096, seed=2)
    file = oracle_lib.compress_image(frame, tile)
    st, rec, out, _ = gpu_decode(file)
    assert st == Status.success and rec == (0, 0, frame.nbytes)
    assert np.array_equal(out[:frame.nbytes].view(np.uint16).reshape(frame.shape), frame)


def test_field_frame_full_size(cuda_ready, oracle_lib):
    frame = workloads.field_frame(4096, 4096, seed=3)
    file = oracle_lib.compress_image(frame, (128, 32))
    st, rec, out, _ = gpu_decode(file)
    assert st == Status.success and rec == (0, 0, frame.nbytes)
    assert np.array_equal(out[:frame.nbytes].view(np.uint32).reshape(frame.shape), frame)


def test_more_than_4096_tiles_and_mixed_geometry(cuda_ready, oracle_lib):
    frames = [workloads.detector_frame(2000, 2100, seed=11), workloads.detector_frame(333, 4097, 12),
              workloads.detector_frame(5000, 70, seed=13)]
    items, keep, expect = [], [], []
    for frame, tile in zip(frames, api.TILE_SHAPES):
        file = oracle_lib.compress_image(frame, tile)
        src, meta, dev = parsed_source(file)
        h, w = frame.shape
        out = device_bytes(frame.nbytes)
        items.append(decode_item(src, api.PixelType.uint16, out, w, h, w * 2))
        keep += [meta, dev, out]
        expect.append((out, frame))
    run = Run(cuda.Operation.decompress, items, keep=keep)
    assert run.status == Status.success
    spec = run.plan.workspace_spec()
    assert (spec.tile.width, spec.tile.height) == (64, 64)  # mixed geometries
    assert run.execute(cuda.decompress_async) == Status.success
    for (out, frame), rec in zip(expect, run.records()):
        assert rec == (0, 0, frame.nbytes)
        assert np.array_equal(host(out)[:frame.nbytes].view(np.uint16).reshape(frame.shape), frame)


def test_staged_tiles_in_reverse_order_with_poisoned_bytes(cuda_ready, oracle_lib):
    """Only the tiles that intersect the ROI are staged, in a fresh buffer in reverse order,
    and the bytes around them are poisoned (reference cuda_decoder_test.cpp:40-82,218)."""
    frame = workloads.detector_frame(700, 300, seed=5)
    file = oracle_lib.compress_image(frame, (64, 64))
    st, meta = api.parse_metadata(file)
    tiles = meta.tiles
    across = -(-700 // 64)
    roi = (100, 50, 333, 170)
    sel = [r * across + c for r in range(50 // 64, (50 + 170 - 1) // 64 + 1)
           for c in range(100 // 64, (100 + 333 - 1) // 64 + 1)]
    stage = bytearray(b"\xee" * 64)
    offsets = {}
    for t in reversed(sel):
        offsets[t] = len(stage)
        stage += file[tiles[t]["offset"]:tiles[t]["offset"] + tiles[t]["length"]]
        stage += b"\xee" * 12
    dev = to_device(np.frombuffer(bytes(stage), dtype=np.uint8))
    maps = (TileMapping * len(sel))(*[TileMapping(t, offsets[t]) for t in sel])
    src = CompressedInput()
    src.bytes = ConstBytes(dev.data_ptr(), len(stage))
    src.metadata = meta.handle
    src.mappings = maps
    src.mapping_count = len(sel)
    out = device_bytes(roi[2] * roi[3] * 2)
    item = decode_item(src, api.PixelType.uint16, out, roi[2], roi[3], roi[2] * 2, roi)
    run = Run(cuda.Operation.decode_roi, [item], keep=[meta, dev, out, maps])
    assert run.status == Status.success
    assert run.execute(cuda.decode_roi_async) == Status.success
    assert run.records()[0] == (0, 0, roi[2] * roi[3] * 2)
    want = frame[roi[1]:roi[1] + roi[3], roi[0]:roi[0] + roi[2]]
    assert np.array_equal(host(out).view(np.uint16).reshape(roi[3], roi[2]), want)


def test_random_rois_match_crop(cuda_ready, oracle_lib):
    rng = np.random.default_rng(99)
    for ptype in (oracle.UINT16, oracle.FLOAT32):
        frame = (workloads.detector_frame(1000, 600, 21) if ptype == oracle.UINT16
                 else workloads.field_frame(1000, 600, 22))
        for tile in api.TILE_SHAPES:
            file = oracle_lib.compress_image(frame, tile)
            for _ in range(8):
                x, y = int(rng.integers(0, 1000)), int(rng.integers(0, 600))
                w, h = int(rng.integers(1, 1001 - x)), int(rng.integers(1, 601 - y))
                st, rec, out, pitch = gpu_decode(file, roi=(x, y, w, h))
                s = frame.itemsize
                assert st == Status.success and rec == (0, 0, w * h * s)
                want = frame[y:y + h, x:x + w]
                assert np.array_equal(out[:want.nbytes].view(frame.dtype).reshape(h, w), want)
