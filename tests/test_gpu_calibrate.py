"""Calibration parity: y = RN(RN(x - offset) * gain) in binary32 (docs/numerical-analysis.md).
Standalone and fused results must equal the host two-rounding form bit for bit except NaN
payloads, equal each other bit for bit (NaNs included), and stay within 1.5 ulp of the FP64
reference for normal results (reference tests/cuda_calibration_test.cpp:121-135,208,328-389,
tests/numerics/support.h:52-57)."""
import json
import os

import numpy as np
import pytest

import oracle
from support import Run, decode_item, device_bytes, host, parsed_source, to_device
from tilestream_b200 import api, cuda, workloads
from tilestream_b200.api import BatchItem, Calibration, Status

pytestmark = pytest.mark.gpu

SPECIAL = np.array([0x00000000, 0x80000000, 0x00000001, 0x80000001, 0x007fffff, 0x00800000,
                    0x80800000, 0x7f7fffff, 0xff7fffff, 0x7f800000, 0xff800000, 0x7fc00000,
                    0xffc00001, 0x7f800001, 0x3f800000, 0x3f800001, 0xbf800000, 0x4b800000,
                    0x33800000, 0x0c000000, 0x72000000], dtype=np.uint32)


def same_bits_or_both_nan(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    fa, fb = a.view(np.float32), b.view(np.float32)
    return (a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(fa) & np.isnan(fb))


def host_form(samples, offset, gain):
    """Two binary32 roundings with numpy (no FMA): the reference host form."""
    x = samples.astype(np.float32) if samples.dtype == np.uint16 else samples.view(np.float32)
    with np.errstate(all="ignore"):
        d = (x - np.float32(offset) if np.ndim(offset) == 0 else x - offset).astype(np.float32)
        return (d * (np.float32(gain) if np.ndim(gain) == 0 else gain)).astype(np.float32)


def calibration(offset, gain, keep):
    cal = Calibration()
    for which, value in (("offset", offset), ("gain", gain)):
        p = getattr(cal, which)
        if np.ndim(value) == 0:
            p.kind = cuda.ParameterKind.scalar
            p.scalar = float(value)
        else:
            arr = np.ascontiguousarray(value, dtype=np.float32)
            dev = to_device(arr)
            keep.append(dev)
            h, w = arr.shape
            p.kind = cuda.ParameterKind.map
            p.map = api.const_view(dev, 2, w, h, w * 4, dev.numel())
    return cal


def gpu_calibrate(samples, offset, gain, in_pitch=None, out_pitch=None):
    h, w = samples.shape
    ptype = 1 if samples.dtype == np.uint16 else 2
    s = samples.itemsize
    in_pitch = in_pitch or w * s
    buf = np.zeros(in_pitch * h, dtype=np.uint8)
    for y in range(h):
        buf[y * in_pitch:y * in_pitch + w * s] = samples[y].view(np.uint8)
    dev = to_device(buf)
    out_pitch = out_pitch or w * 4
    out = device_bytes(out_pitch * h)
    keep = [dev, out]
    item = BatchItem()
    item.input = api.const_view(dev, ptype, w, h, in_pitch, dev.numel())
    item.output = api.view(out, 2, w, h, out_pitch, out.numel())
    item.calibration = calibration(offset, gain, keep)
    run = Run(cuda.Operation.calibrate, [item], keep=keep)
    assert run.status == Status.success
    assert run.execute(cuda.calibrate_async) == Status.success
    assert run.records()[0] == (0, 0, w * h * 4)
    o = host(out)
    return np.stack([o[y * out_pitch:y * out_pitch + 4 * w].view(np.uint32) for y in range(h)])


def test_standalone_matches_host_form(cuda_ready):
    rng = np.random.default_rng(5)
    u16 = rng.integers(0, 65536, (123, 517), dtype=np.uint16)
    f32 = workloads.field_frame(517, 123, seed=8)
    off = rng.normal(100, 5, (123, 517)).astype(np.float32)
    gain = rng.uniform(0.9, 1.1, (123, 517)).astype(np.float32)
    for samples in (u16, f32):
        for o, g in ((100.0, 1.05), (off, 1.05), (100.0, gain), (off, gain)):
            got = gpu_calibrate(samples, o, g)
            want = host_form(samples, o, g).view(np.uint32)
            assert np.all(same_bits_or_both_nan(got, want))
            got2 = gpu_calibrate(samples, o, g, in_pitch=samples.itemsize * 520, out_pitch=4 * 521)
            assert np.array_equal(got, got2)


def test_special_word_grid(cuda_ready):
    n = SPECIAL.size
    idx = np.arange(n ** 3)
    x = SPECIAL[idx % n].reshape(n * n, n)
    o = SPECIAL[idx // n % n].view(np.float32).reshape(n * n, n)
    g = SPECIAL[idx // n // n].view(np.float32).reshape(n * n, n)
    got = gpu_calibrate(x, o, g)
    want = host_form(x, o, g).view(np.uint32)
    assert np.all(same_bits_or_both_nan(got, want))


def test_every_uint16_value_within_bound(cuda_ready, oracle_lib):
    x = np.arange(65536, dtype=np.uint16).reshape(128, 512)
    got = gpu_calibrate(x, 100.0, 1.05).view(np.float32)
    ref = (x.astype(np.float64) - np.float64(np.float32(100.0))) * np.float64(np.float32(1.05))
    ulp = np.spacing(np.abs(ref).astype(np.float32)).astype(np.float64)
    err = np.abs(got.astype(np.float64) - ref) / ulp
    normal = np.abs(ref) >= 2.0 ** -126
    assert err[normal].max() <= 1.5 + 2.0 ** -20
    assert np.all(same_bits_or_both_nan(got.view(np.uint32),
                                        host_form(x, 100.0, 1.05).view(np.uint32)))


@pytest.mark.parametrize("ptype", [1, 2])
def test_fused_equals_separate(cuda_ready, oracle_lib, ptype):
    """decode_calibrate == decode then calibrate, bit for bit, over a full image and an ROI."""
    frame = (workloads.detector_frame(1100, 700, 51) if ptype == 1
             else workloads.field_frame(1100, 700, 52))
    for tile in api.TILE_SHAPES:
        file = oracle_lib.compress_image(frame, tile)
        for roi in ((0, 0, 1100, 700), (131, 77, 555, 401)):
            x, y, w, h = roi
            off, gain = workloads.calibration_maps(w, h, seed=roi[0] + 1)
            src, meta, dev = parsed_source(file)
            keep = [meta, dev]
            cal = calibration(off, np.float32(1.05) if roi[0] else gain, keep)
            out = device_bytes(w * h * 4)
            keep.append(out)
            item = decode_item(src, 2, out, w, h, w * 4, roi, cal)
            run = Run(cuda.Operation.decode_calibrate, [item], keep=keep)
            assert run.status == Status.success
            assert run.execute(cuda.decode_calibrate_async) == Status.success
            assert run.records()[0] == (0, 0, w * h * 4)
            fused = host(out).view(np.uint32).reshape(h, w)
            region = frame[y:y + h, x:x + w]
            separate = gpu_calibrate(region, off, np.float32(1.05) if roi[0] else gain)
            assert np.array_equal(fused, separate), (tile, roi)


def contract_rows():
    with open(os.path.join(os.path.dirname(__file__), "golden",
                           "calibration_contract_rows.json")) as f:
        return json.load(f)


def fused(oracle_lib, samples, offset, gain):
    """decode_calibrate of a one-row archive of `samples` with per-pixel maps."""
    h, w = samples.shape
    src, meta, dev = parsed_source(oracle_lib.compress_image(samples))
    keep = [meta, dev]
    cal = calibration(offset, gain, keep)
    out = device_bytes(w * h * 4)
    keep.append(out)
    item = decode_item(src, 2, out, w, h, w * 4, (0, 0, w, h), cal)
    run = Run(cuda.Operation.decode_calibrate, [item], keep=keep)
    assert run.status == Status.success
    assert run.execute(cuda.decode_calibrate_async) == Status.success
    assert run.records()[0] == (0, 0, w * h * 4)
    return host(out).view(np.uint32).reshape(h, w)


def test_special_value_contract(cuda_ready, oracle_lib):
    """The reference's 42 special-value contract rows with their exact expected words
    (tests/numerics/support.h:404-456; NaN results compare by class), through every path the
    reference runs them on (tests/cuda_numerics_test.cpp:161-200): per-pixel maps standalone
    and fused, the rows whose sample is a uint16 value as uint16 samples standalone and fused,
    and one 1x1 image per row with scalar parameters."""
    rows = contract_rows()
    word = lambda key, sel=rows: np.array([[int(r[key], 16) for r in sel]],  # noqa: E731
                                          np.uint32)
    as_f32 = lambda a: a.view(np.float32)  # noqa: E731

    def check(got, sel, path):
        want = word("expected", sel)
        assert np.all(same_bits_or_both_nan(got, want)), (
            path, [r["note"] for r, ok in zip(sel, same_bits_or_both_nan(got, want)[0]) if not ok])

    x, o, g = word("x"), as_f32(word("offset")), as_f32(word("gain"))
    check(gpu_calibrate(x, o, g), rows, "maps")
    check(fused(oracle_lib, x, o, g), rows, "fused")

    def is_uint16(r):
        v = np.uint32(int(r["x"], 16)).view(np.float32)
        return bool(0 <= v <= 65535 and v == np.floor(v) and not np.signbit(v))

    ints = [r for r in rows if is_uint16(r)]
    assert len(ints) >= 10
    xi = as_f32(word("x", ints)).astype(np.uint16)
    oi, gi = as_f32(word("offset", ints)), as_f32(word("gain", ints))
    check(gpu_calibrate(xi, oi, gi), ints, "uint16")
    check(fused(oracle_lib, xi, oi, gi), ints, "uint16 fused")

    items, outs, keep = [], [], []
    for r in rows:
        inp = to_device(np.array([int(r["x"], 16)], np.uint32).view(np.uint8))
        out = device_bytes(4)
        outs.append(out)
        keep += [inp, out]
        item = BatchItem()
        item.input = api.const_view(inp, 2, 1, 1, 4, 4)
        item.output = api.view(out, 2, 1, 1, 4, 4)
        item.calibration = calibration(np.uint32(int(r["offset"], 16)).view(np.float32),
                                       np.uint32(int(r["gain"], 16)).view(np.float32), keep)
        items.append(item)
    run = Run(cuda.Operation.calibrate, items, keep=keep)
    assert run.status == Status.success
    assert run.execute(cuda.calibrate_async) == Status.success
    assert all(rec == (0, 0, 4) for rec in run.records())
    check(np.array([[host(out).view(np.uint32)[0] for out in outs]]), rows, "scalars")
