"""The library's host codec (tilestream::cpu::compress/decompress) against the oracle, in the
manner of the reference tests/cpu_codec_test.cpp and fp32_codec_test.cpp."""
import json
import os

import numpy as np
import pytest

import oracle
from tilestream_b200 import api, cpu, workloads
from tilestream_b200.api import ParseLimits, Status, TileShape

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def read_hex(name):
    with open(os.path.join(GOLDEN, name + ".hex")) as f:
        return bytes(int(t, 16) for t in f.read().split())


def encode(buf, ptype, w, h, pitch, tile=(128, 32), capacity=None, extra=16):
    st, bound = api.compress_bound(api.image_spec(ptype, w, h), TileShape(*tile))
    assert st == Status.success
    out = np.full(bound + extra, 0xA5, dtype=np.uint8)
    st, n = cpu.compress(api.const_view(buf, ptype, w, h, pitch, capacity), TileShape(*tile),
                         api.mutable_bytes(out, bound))
    assert st == Status.success, st
    assert np.all(out[n:] == 0xA5) if n < bound else True
    return out[:n].tobytes()


def decode(file, ptype, w, h, pitch=None, fill=0xA5, limits=None):
    s = api.sample_bytes(ptype)
    pitch = pitch or w * s
    out = np.full(pitch * h, fill, dtype=np.uint8)
    src = np.frombuffer(file, dtype=np.uint8)
    st = cpu.decompress(api.const_bytes(src), api.view(out, ptype, w, h, pitch), limits)
    return st, out


def test_golden_files():
    for name, c in json.load(open(os.path.join(GOLDEN, "cases.json"))).items():
        dtype = np.uint16 if c["type"] == 1 else np.uint32
        px = np.array(c["pixels"], dtype=dtype)
        file = read_hex(name)
        assert encode(px, c["type"], c["width"], c["height"], c["width"] * px.itemsize) == file
        st, out = decode(file, c["type"], c["width"], c["height"])
        assert st == Status.success and np.array_equal(out.view(dtype), px)


def test_seeded_cases_against_oracle(oracle_lib):
    for seed in range(13000000, 13000000 + 2000):
        c = oracle_lib.case(seed)
        file = encode(c["bytes"], c["type"], c["width"], c["height"], c["pitch"], c["tile"])
        assert file == oracle_lib.compress(c["bytes"], c["type"], c["width"], c["height"],
                                           c["pitch"], c["tile"]), seed
        st, out = decode(file, c["type"], c["width"], c["height"], c["pitch"], fill=0x5A)
        assert st == Status.success and np.array_equal(out, c["bytes"]), seed


@pytest.mark.parametrize("tile", api.TILE_SHAPES)
def test_detector_frame(oracle_lib, tile):
    frame = workloads.detector_frame(1024, 1024, seed=1)
    file = encode(frame, 1, 1024, 1024, 2048, tile)
    assert file == oracle_lib.compress_image(frame, tile)
    st, out = decode(file, 1, 1024, 1024)
    assert st == Status.success and np.array_equal(out.view(np.uint16).reshape(1024, 1024), frame)


def test_field_frame_special_words(oracle_lib):
    frame = workloads.field_frame(700, 300, seed=3)
    for tile in api.TILE_SHAPES:
        file = encode(frame, 2, 700, 300, 2800, tile)
        assert file == oracle_lib.compress_image(frame, tile)
        st, out = decode(file, 2, 700, 300)
        assert st == Status.success and np.array_equal(out.view(np.uint32).reshape(300, 700),
                                                       frame)


def _dataset_fixtures():
    from golden import inputs
    yield from inputs.datasets()


def test_dataset_fixtures_match_reference(oracle_lib, reference):
    """The reference's image fixtures (datasets/fixtures/*.npy: a CT slice, an elevation field
    and two generated images, copied into tests/golden/datasets by make_golden.py): for every tile shape the library's
    encoder, the oracle and the reference build emit the same bytes, and the file decodes back
    to the same words."""
    seen = 0
    for name, img in _dataset_fixtures():
        assert img.ndim == 2 and img.dtype in (np.uint16, np.float32), name
        words = np.ascontiguousarray(img if img.dtype == np.uint16 else img.view(np.uint32))
        ptype = 1 if words.dtype == np.uint16 else 2
        h, w = words.shape
        for tile in api.TILE_SHAPES:
            file = encode(words, ptype, w, h, w * words.itemsize, tile)
            assert file == oracle_lib.compress_image(words, tile), (name, tile)
            assert file == reference.compress_image(words, tile), (name, tile)
            st, out = decode(file, ptype, w, h)
            assert st == Status.success, (name, tile)
            assert np.array_equal(out.view(words.dtype).reshape(h, w), words), (name, tile)
        seen += 1
    assert seen >= 2


def test_every_uint16_value(oracle_lib):
    img = np.arange(65536, dtype=np.uint16).reshape(256, 256)[:, ::-1].copy()
    file = encode(img, 1, 256, 256, 512)
    assert file == oracle_lib.compress_image(img)
    st, out = decode(file, 1, 256, 256)
    assert np.array_equal(out.view(np.uint16).reshape(256, 256), img)


def test_invalid_views_leave_outputs_untouched():
    """Each rejected call returns its documented status and writes nothing."""
    px = np.arange(64, dtype=np.uint16)
    out = np.full(4096, 0x77, dtype=np.uint8)
    good = api.const_view(px, 1, 8, 8, 16)
    cases = [
        (api.const_view(px, 3, 8, 8, 16), Status.unsupported_type),
        (api.const_view(px, 1, 0, 8, 16), Status.invalid_argument),
        (api.const_view(px, 1, 8, 8, 14), Status.invalid_argument),   # pitch < row
        (api.const_view(px, 1, 8, 8, 17), Status.invalid_argument),   # pitch % 2
        (api.const_view(px, 1, 8, 8, 16, capacity=100), Status.buffer_too_small),
        (api.ConstImageView(0, api.image_spec(1, 8, 8), 16, 128), Status.invalid_argument),
        (api.ConstImageView(px.ctypes.data + 1, api.image_spec(1, 8, 8), 16, 127),
         Status.invalid_argument),                                    # misaligned
    ]
    for view, want in cases:
        st, n = cpu.compress(view, TileShape(), api.mutable_bytes(out))
        assert st == want and np.all(out == 0x77)
    st, n = cpu.compress(good, TileShape(64, 32), api.mutable_bytes(out))
    assert st == Status.invalid_argument and np.all(out == 0x77)
    st, n = cpu.compress(good, TileShape(), api.mutable_bytes(out, 100))
    assert st == Status.buffer_too_small and np.all(out == 0x77)
    # Overlapping input and output.
    both = np.zeros(8192, dtype=np.uint8)
    st, n = cpu.compress(api.const_view(both, 1, 8, 8, 16, 128), TileShape(),
                         api.mutable_bytes(both))
    assert st == Status.invalid_argument


def test_decompress_rejects_mismatched_output(oracle_lib):
    frame = workloads.detector_frame(100, 50, seed=9)
    file = oracle_lib.compress_image(frame)
    for w, h, t in ((101, 50, 1), (100, 49, 1), (100, 50, 2)):
        st, out = decode(file, t, w, h)
        assert st == Status.invalid_argument and np.all(out == 0xA5)
    st, out = decode(file, 1, 100, 50, limits=ParseLimits(100, 2 ** 63 - 1, 2 ** 63 - 1))
    assert st == Status.resource_limit


def test_pitched_output_padding_untouched(oracle_lib):
    frame = workloads.detector_frame(129, 33, seed=10)
    file = oracle_lib.compress_image(frame)
    st, out = decode(file, 1, 129, 33, pitch=129 * 2 + 6)
    assert st == Status.success
    rows = out.reshape(33, 264)
    assert np.all(rows[:, 258:] == 0xA5)
    assert np.array_equal(rows[:, :258].copy().view(np.uint16), frame)
