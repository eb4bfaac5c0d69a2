"""Pins the C oracle: it must reproduce the reference's golden files and agree byte for byte with
the reference CPU codec itself (compiled from its sources into oracle/_ref) on the reference's
seeded robustness cases and on the C1 round trip."""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
from tilestream_b200 import workloads

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def read_hex(name):
    with open(os.path.join(GOLDEN, name + ".hex")) as f:
        return bytes(int(t, 16) for t in f.read().split())


def golden_cases():
    with open(os.path.join(GOLDEN, "cases.json")) as f:
        return json.load(f)


def test_golden_files(oracle_lib):
    """Hand-calculated golden bitstreams (reference tests/cpu_codec_test.cpp:83-119,
    fp32_codec_test.cpp:81-90): encode reproduces them, decode returns the pixels, and the
    parser reports the expected tile mode."""
    for name, c in golden_cases().items():
        dtype = np.uint16 if c["type"] == 1 else np.uint32
        px = np.array(c["pixels"], dtype=dtype)
        file = read_hex(name)
        assert oracle_lib.compress(px, c["type"], c["width"], c["height"],
                                   c["width"] * px.itemsize) == file, name
        st, out = oracle_lib.decompress(file, c["type"], c["width"], c["height"])
        assert st == 0 and np.array_equal(out.view(dtype), px), name
        st, meta = oracle_lib.parse(file)
        assert st == 0 and len(meta["tiles"]) == 1 and meta["tiles"][0]["mode"] == c["mode"]


def test_golden_files_match_reference_checkout():
    """The committed fixtures equal the reference's own golden files (when present)."""
    if oracle.reference_dir() is None:
        pytest.skip("TILESTREAM_REFERENCE does not name the reference checkout")
    ref_dir = os.path.join(oracle.reference_dir(), "tests", "golden")
    for name in golden_cases():
        with open(os.path.join(ref_dir, name + ".hex")) as f:
            upstream = bytes(int(t, 16) for t in f.read().split())
        assert read_hex(name) == upstream, name


def contract_rows():
    with open(os.path.join(GOLDEN, "calibration_contract_rows.json")) as f:
        return json.load(f)


def same_word(got, want):
    """Equal words, or both NaN (NaN results compare by class)."""
    nan = lambda w: (w & 0x7f800000) == 0x7f800000 and (w & 0x007fffff) != 0  # noqa: E731
    return got == want or (nan(got) and nan(want))


def test_calibration_contract_rows(oracle_lib):
    """The reference's special-value contract (tests/numerics/support.h:404-456, run on the host
    form by tests/numerics_test.cpp:79-87): the oracle's two-rounding form gives each row's
    exact word."""
    rows = contract_rows()
    assert len(rows) == 42
    words = lambda k: np.array([[int(r[k], 16) for r in rows]], np.uint32)  # noqa: E731
    got = oracle_lib.calibrate_image(words("x"), words("offset").view(np.float32),
                                     words("gain").view(np.float32)).view(np.uint32)[0]
    for r, g in zip(rows, got):
        assert same_word(int(g), int(r["expected"], 16)), (r["note"], hex(int(g)))


def test_calibration_contract_rows_match_reference_checkout():
    """The committed rows equal the reference header's table (when present)."""
    if oracle.reference_dir() is None:
        pytest.skip("TILESTREAM_REFERENCE does not name the reference checkout")
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    assert mod.contract_rows() == contract_rows()


def test_format_worked_example(oracle_lib):
    """docs/format.md:77: three 3-bit residuals [1, 2, 7] pack to the word 0x000001d1. A row
    100, 99, 100, 96, 96, ... has deltas -1, +1, -4 (zigzag 1, 2, 7) followed by zeros."""
    row = np.array([100, 99, 100, 96] + [96] * 124, dtype=np.uint16)
    file = oracle_lib.compress_image(np.tile(row, (4, 1)))
    st, meta = oracle_lib.parse(file)
    assert st == 0 and meta["tiles"][0]["mode"] == oracle.PREDICT
    seg = meta["segments"][0]
    assert seg["bit_width"] == 3
    off = int(meta["tiles"][0]["offset"] + seg["payload_offset"])
    assert file[off:off + 4] == bytes([0xd1, 0x01, 0x00, 0x00])


def test_bound_examples(oracle_lib):
    """docs/format.md:132."""
    assert oracle_lib.compress_bound(1, 1, 1) == (0, 100)
    assert oracle_lib.compress_bound(2, 1, 1) == (0, 100)
    assert oracle_lib.compress_bound(1, 128, 32) == (0, 8288)
    assert oracle_lib.compress_bound(1, 129, 33) == (0, 8708)


def test_seeded_cases_match_reference(oracle_lib, reference):
    for seed in range(13000000, 13000000 + 1500):
        c = oracle_lib.case(seed)
        args = (c["bytes"], c["type"], c["width"], c["height"], c["pitch"], c["tile"])
        a = oracle_lib.compress(*args)
        assert a == reference.compress(*args), seed
        st1, o1 = oracle_lib.decompress(a, c["type"], c["width"], c["height"], c["pitch"],
                                        fill=0x5a)
        st2, o2 = reference.decompress(a, c["type"], c["width"], c["height"], c["pitch"],
                                       fill=0x5a)
        assert st1 == st2 == 0 and np.array_equal(o1, o2) and np.array_equal(o1, c["bytes"])


def test_c1_golden_round_trip(oracle_lib):
    """Config 1: uint16 1024x1024 frame, seed 1, tiles 128x32; the bitstream equals the
    reference encoding recorded in c1_roundtrip.json, and decodes back bit-exactly."""
    with open(os.path.join(GOLDEN, "c1_roundtrip.json")) as f:
        want = json.load(f)
    frame = workloads.detector_frame(1024, 1024, seed=1)
    assert hashlib.sha256(frame.tobytes()).hexdigest() == want["pixels_sha256"]
    file = oracle_lib.compress_image(frame, (128, 32))
    assert len(file) == want["file_bytes"]
    assert hashlib.sha256(file).hexdigest() == want["file_sha256"]
    assert np.array_equal(oracle_lib.decompress_image(file), frame)


def test_parser_statuses_match_reference(oracle_lib, reference):
    """Seeded structural mutations of valid files: the oracle parser returns the reference
    parser's status for every mutant (with the fuzz harness budgets)."""
    rng = np.random.default_rng(17)
    for seed in range(13000000, 13000000 + 150):
        c = oracle_lib.case(seed)
        file = bytearray(oracle_lib.compress(c["bytes"], c["type"], c["width"], c["height"],
                                             c["pitch"], c["tile"]))
        for _ in range(12):
            m = bytearray(file)
            kind = rng.integers(0, 4)
            if kind == 0 and len(m):
                m[int(rng.integers(0, min(len(m), 200)))] ^= int(rng.integers(1, 256))
            elif kind == 1 and len(m):
                m[int(rng.integers(0, len(m)))] ^= int(rng.integers(1, 256))
            elif kind == 2:
                m = m[:int(rng.integers(0, len(m) + 1))]
            else:
                m += bytes(int(rng.integers(1, 9)))
            a, _ = oracle_lib.parse(bytes(m), oracle.FUZZ_LIMITS)
            b, _ = reference.parse(bytes(m), oracle.FUZZ_LIMITS)
            assert a == b, (seed, kind)
