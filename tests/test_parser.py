"""The library's untrusted-file parser: statuses and tables against the oracle on truncations,
field mutations and the reference's fuzz corpora (reference tests/cpu_codec_test.cpp:367-510,
fuzz/harness.h, fuzz/corpus)."""
import os

import numpy as np
import pytest

import oracle
from tilestream_b200 import api, cpu, workloads
from tilestream_b200.api import ParseLimits, Status

LIMITS = ParseLimits(*oracle.FUZZ_LIMITS)


def ours(file, limits=None):
    st, meta = api.parse_metadata(np.frombuffer(file, dtype=np.uint8) if file else b"",
                                  limits, size=len(file))
    return int(st), meta


def same_tables(meta, ref_meta):
    t = meta.tiles
    s = meta.segments
    assert meta.file_bytes == ref_meta["file_bytes"]
    assert (meta.image.type, meta.image.width, meta.image.height) == (
        ref_meta["type"], ref_meta["width"], ref_meta["height"])
    assert (meta.tile.width, meta.tile.height) == tuple(ref_meta["tile"])
    assert np.array_equal(t.view(np.uint8), ref_meta["tiles"].view(np.uint8))
    assert np.array_equal(s.view(np.uint8), ref_meta["segments"].view(np.uint8))


def check(o, file, limits=LIMITS):
    st, meta = ours(file, limits)
    want, ref_meta = o.parse(file, oracle.FUZZ_LIMITS if limits is LIMITS else None)
    assert st == want, (st, want)
    if st == 0:
        same_tables(meta, ref_meta)
    return st


def test_valid_files_tables_match(oracle_lib):
    for seed in range(13000000, 13000300):
        c = oracle_lib.case(seed)
        file = oracle_lib.compress(c["bytes"], c["type"], c["width"], c["height"], c["pitch"],
                                   c["tile"])
        assert check(oracle_lib, file, None) == 0


def test_large_files_tables_match_reference(oracle_lib, reference):
    """4096x4096 frames (4096 tiles each): the payloads are checked in ranges of tiles on
    several host threads; the tables must equal the reference parser's, and a bad row in the
    last tile must still be found."""
    frame = workloads.detector_frame(4096, 4096, seed=2)
    for tile in api.TILE_SHAPES:
        file = oracle_lib.compress_image(frame, tile)
        st, meta = ours(file)
        want, ref_meta = reference.parse(file)
        assert st == want == 0
        same_tables(meta, ref_meta)
        tiles, segments = meta.tiles, meta.segments
        last = len(tiles) - 1
        assert int(tiles["mode"][last]) == 2
        seg = segments[int(tiles["first_segment"][last]) + int(tiles["height"][last]) - 1]
        bad = bytearray(file)
        bad[int(tiles["offset"][last]) + int(seg["payload_offset"]) - 8 + 6] = 0x40
        assert ours(bytes(bad))[0] == reference.parse(bytes(bad))[0] == int(Status.malformed_data)


def test_every_truncation(oracle_lib):
    frame = workloads.detector_frame(300, 70, seed=4)
    file = oracle_lib.compress_image(frame, (64, 64))
    for n in range(0, len(file)):
        assert check(oracle_lib, file[:n]) != 0
    assert check(oracle_lib, file) == 0


def test_every_header_and_entry_byte(oracle_lib):
    """Flip each header and index byte (and a few payload bytes) of small files."""
    for seed in (13000000, 13000001, 13000004, 13000007, 13000010):
        c = oracle_lib.case(seed)
        file = bytearray(oracle_lib.compress(c["bytes"], c["type"], c["width"], c["height"],
                                             c["pitch"], c["tile"]))
        stop = min(len(file), 64 + 32 * 6 + 64)
        for i in range(stop):
            for x in (0x01, 0x80, 0xFF):
                m = bytearray(file)
                m[i] ^= x
                check(oracle_lib, bytes(m))


def test_other_format_versions_are_unsupported(oracle_lib):
    """Only version 1.0 is defined; any other major or minor version (a v1.1 file included) is
    unsupported, not guessed (reference docs/format.md:16-17,32)."""
    frame = workloads.detector_frame(130, 70, seed=8)
    file = oracle_lib.compress_image(frame)
    assert check(oracle_lib, file) == 0
    for major, minor in ((1, 1), (1, 0xFFFF), (2, 0), (0, 0), (0, 1)):
        m = bytearray(file)
        m[8:10] = major.to_bytes(2, "little")
        m[10:12] = minor.to_bytes(2, "little")
        assert check(oracle_lib, bytes(m)) == int(Status.unsupported_format)


def test_seeded_mutation_campaign(oracle_lib):
    rng = np.random.default_rng(2026)
    for seed in range(13000000, 13000400):
        c = oracle_lib.case(seed)
        file = oracle_lib.compress(c["bytes"], c["type"], c["width"], c["height"], c["pitch"],
                                   c["tile"])
        for _ in range(6):
            m = bytearray(file)
            for _ in range(int(rng.integers(1, 4))):
                if len(m) == 0:
                    break
                at = int(rng.integers(0, len(m)))
                m[at] = int(rng.integers(0, 256))
            check(oracle_lib, bytes(m))


def test_limits(oracle_lib):
    frame = workloads.detector_frame(300, 200, seed=6)
    file = oracle_lib.compress_image(frame)
    big = 2 ** 63 - 1
    for lim in ((len(file) - 1, big, big), (big, 11, big), (big, big, 72 + 32 * 12),
                (big, big, 72 + 32 * 12 + 24 * 10)):
        st, _ = ours(file, ParseLimits(*lim))
        want, _ = oracle_lib.parse(file, lim)
        assert st == want == int(Status.resource_limit)
    st, _ = ours(file, ParseLimits(len(file), 21, big))  # 3 x 7 tiles of 128x32
    assert st == 0


def test_malformed_payload_outranks_segment_budget(oracle_lib, reference):
    """A file over the row-segment budget whose payload is also malformed reports
    malformed_data: every payload is checked before that budget (reference
    src/cpu/parser.cpp:86-171 walks the payloads before it sizes the segment table)."""
    frame = workloads.detector_frame(300, 200, seed=6)
    file = oracle_lib.compress_image(frame)
    st, meta = ours(file)
    assert st == 0
    tiles, segments = meta.tiles, meta.segments
    predict = [i for i in range(len(tiles)) if int(tiles["mode"][i]) == 2]
    last = predict[-1]
    # A segment's payload_offset is that of its packed words, just after its 8-byte descriptor.
    seg = segments[int(tiles["first_segment"][last])]
    desc = int(tiles["offset"][last]) + int(seg["payload_offset"]) - 8
    bad = bytearray(file)
    bad[desc + 5] = 1  # a reserved byte of the last PREDICT tile's first row descriptor
    big = 2 ** 63 - 1
    # Room for the 21 tile records (72 + 32 * 21 bytes) but not for the file's row segments.
    tight = (big, big, 72 + 32 * 21 + 24 * 10)
    for candidate, want in ((file, Status.resource_limit), (bytes(bad), Status.malformed_data)):
        got, _ = ours(candidate, ParseLimits(*tight))
        assert got == int(want)
        assert oracle_lib.parse(candidate, tight)[0] == int(want)
        assert reference.parse(candidate, tight)[0] == int(want)


def test_empty_and_null_sources():
    st, _ = ours(b"")
    assert st == int(Status.malformed_data)
    h = api.ConstBytes(0, 10)
    import ctypes as C
    from tilestream_b200 import _native as N
    out = C.c_void_p(0)
    assert N.lib().ts_parse_metadata(h, None, C.byref(out)) == int(Status.invalid_argument)


def _corpus(kind):
    from golden import inputs
    yield from inputs.corpus(kind)


def test_parse_corpus_replay(oracle_lib, reference):
    """Every input of the reference parse corpus: our parser's status and tables equal the
    reference parser's, and accepted files decode to the reference's pixels."""
    n = 0
    for name, data in _corpus("parse"):
        st, meta = ours(data, LIMITS)
        want, ref_meta = reference.parse(data, oracle.FUZZ_LIMITS)
        assert st == want, name
        if st == 0:
            same_tables(meta, ref_meta)
            t, w, h = ref_meta["type"], ref_meta["width"], ref_meta["height"]
            if w * h * oracle.SAMPLE[t] <= 4 << 20:
                out = np.full(w * h * oracle.SAMPLE[t], 0xA5, np.uint8)
                assert cpu.decompress(api.const_bytes(np.frombuffer(data, np.uint8)),
                                      api.view(out, t, w, h), LIMITS) == Status.success
                rs, rout = reference.decompress(data, t, w, h, limits=oracle.FUZZ_LIMITS)
                assert rs == 0 and np.array_equal(out, rout), name
        n += 1
    assert n > 100


def test_mutation_corpus_replay(oracle_lib, reference):
    """Every input of the reference mutation corpus rebuilt into its mutated file
    (fuzz/harness.h:227-290): statuses and tables equal the reference parser's."""
    n = 0
    for name, data in _corpus("mutation"):
        file = oracle_lib.mutation_file(data)
        if file is None:
            continue
        st, meta = ours(file, LIMITS)
        want, ref_meta = reference.parse(file, oracle.FUZZ_LIMITS)
        assert st == want, name
        if st == 0:
            same_tables(meta, ref_meta)
        n += 1
    assert n > 300
