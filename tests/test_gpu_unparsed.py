"""Decode of .tsc files never parsed on the host (decode_unparsed_async): the host checks the
header, the decoder validates the index, payloads and rows on the device with the parser's
rules. Checked against the parser and the oracle:

* valid files of both pixel types, every tile shape and ragged sizes (1x1, one-column tiles,
  partial tiles) decode to the oracle's words, several files per launch, pitched outputs, and
  nothing outside each output is written;
* every file of the reference's fuzz corpora (parse, and the mutation corpus rebuilt into its
  files), and 1,200 seeded byte mutations of valid files: the call's status equals
  parse_metadata's for header failures; otherwise the device verdict is success exactly when
  parse_metadata accepts (then the words equal the CPU decode) and malformed_data when it
  rejects, and no write leaves the output's bounds;
* device bytes whose header differs from the host copy are malformed; the host's argument
  checks.
"""
import struct

import numpy as np
import pytest

from support import SENTINEL, device_bytes, host, to_device
from tilestream_b200 import api, cuda, workloads
from tilestream_b200.api import ConstBytes, ResultBuffer, Status

pytestmark = pytest.mark.gpu

GUARD = 256  # sentinel bytes before and after every output


def geometry(file: bytes):
    """(type, width, height) from a header's fields, or None for a file shorter than one."""
    if len(file) < 64:
        return None
    ptype = file[14]
    width, height = struct.unpack_from("<II", file, 16)
    return ptype, width, height


class Batch:
    """Files copied to the device with sentinel-guarded outputs, decoded in one call."""

    def __init__(self, files, pad=0):
        self.files, self.keep, self.outs, self.entries = files, [], [], []
        for k, file in enumerate(files):
            ptype, w, h = geometry(file)
            s = 4 if ptype == 2 else 2
            pitch = (w * s + 15) // 16 * 16 + (pad if k % 2 else 0)
            out = device_bytes(GUARD + pitch * h + GUARD)
            src = to_device(np.frombuffer(file, np.uint8))
            view = api.ImageView(out.data_ptr() + GUARD, api.image_spec(ptype, w, h), pitch,
                                 pitch * h)
            self.keep += [src, out]
            self.outs.append((out, pitch, w, h, s))
            self.entries.append((ConstBytes(src.data_ptr(), len(file)), file[:64], view))
        self.results = device_bytes(16 * max(1, len(files)), fill=0xFF)

    def run(self):
        return cuda.decode_unparsed_async(self.entries,
                                          ResultBuffer(self.results.data_ptr(), len(self.files)))

    def records(self):
        import torch
        torch.cuda.synchronize()
        raw = host(self.results).view(np.uint64).reshape(-1, 2)[:len(self.files)]
        return [(int(r[0]) & 0xFFFFFFFF, int(r[1])) for r in raw]

    def output(self, k):
        out, pitch, w, h, s = self.outs[k]
        buf = host(out)
        assert np.all(buf[:GUARD] == SENTINEL) and np.all(buf[GUARD + pitch * h:] == SENTINEL), k
        rows = buf[GUARD:GUARD + pitch * h].reshape(h, pitch)
        return np.ascontiguousarray(rows[:, :w * s]).reshape(-1), rows[:, w * s:]


def expect_cpu(o, file):
    ptype, w, h = geometry(file)
    st, want = o.decompress(file, ptype, w, h)
    assert st == 0
    return want


def test_valid_files_decode_like_the_oracle(cuda_ready, oracle_lib):
    o = oracle_lib
    cases = [("u16", 4096, 4096, (128, 32)), ("u16", 1, 1, (64, 64)), ("u16", 1, 300, (256, 16)),
             ("u16", 257, 33, (128, 32)), ("f32", 1000, 700, (64, 64)), ("f32", 129, 1, (256, 16)),
             ("u16", 777, 513, (256, 16)), ("f32", 4096, 1024, (128, 32)),
             ("u16", 300, 200, (64, 64))]
    files = []
    for k, (kind, w, h, tile) in enumerate(cases):
        img = (workloads.detector_frame(w, h, seed=70 + k) if kind == "u16"
               else workloads.field_frame(w, h, seed=70 + k))
        files.append(o.compress_image(img, tile))
    for group in (files[:1], files[1:5], files[5:]):  # one file, and several per launch
        b = Batch(group, pad=48)
        assert b.run() == Status.success
        recs = b.records()
        for k, file in enumerate(group):
            ptype, w, h = geometry(file)
            assert recs[k] == (0, w * h * (4 if ptype == 2 else 2)), (k, recs[k])
            got, pad = b.output(k)
            assert np.array_equal(got, np.frombuffer(expect_cpu(o, file), np.uint8)), k
            assert np.all(pad == SENTINEL), k


def verdicts(o, files):
    """Decodes each file alone (one call per file, one synchronization for all) and compares
    with parse_metadata: returns (accepted, rejected) counts."""
    accepted = rejected = 0
    runs = []
    for file in files:
        st_parse, _ = api.parse_metadata(np.frombuffer(file, np.uint8) if file else
                                         np.zeros(1, np.uint8), size=len(file))
        g = geometry(file)
        if g is None or g[0] not in (1, 2) or g[1] * g[2] > (1 << 22) or g[1] * g[2] == 0:
            # The header check fails before any geometry is used: statuses must agree.
            if g is not None and g[1] * g[2] <= (1 << 22):
                src = to_device(np.frombuffer(file, np.uint8))
                out = device_bytes(64)
                view = api.ImageView(out.data_ptr(), api.image_spec(1, 1, 1), 16, 16)
                res = device_bytes(16)
                st = cuda.decode_unparsed_async([(ConstBytes(src.data_ptr(), len(file)),
                                                  file[:64], view)],
                                                ResultBuffer(res.data_ptr(), 1))
                assert st != Status.success and st == st_parse, (st, st_parse)
            continue
        b = Batch([file])
        st = b.run()
        if st != Status.success:
            assert st == st_parse, (st, st_parse)
            rejected += 1
            continue
        runs.append((file, b, st_parse))
    for file, b, st_parse in runs:
        (status, nbytes), = b.records()
        got, pad = b.output(0)
        assert np.all(pad == SENTINEL)
        if st_parse == Status.success:
            assert (status, nbytes) == (0, len(got)), (status, nbytes)
            assert np.array_equal(got, np.frombuffer(expect_cpu(o, file), np.uint8))
            accepted += 1
        else:
            assert st_parse == Status.malformed_data, st_parse
            assert (status, nbytes) == (int(Status.malformed_data), 0), (status, nbytes)
            rejected += 1
    return accepted, rejected


def test_fuzz_corpora_verdicts_match_the_parser(cuda_ready, oracle_lib):
    from golden import inputs
    files = [data for _, data in inputs.corpus("parse")]
    for _, data in inputs.corpus("mutation"):
        f = oracle_lib.mutation_file(data)
        if f is not None:
            files.append(f)
    accepted, rejected = verdicts(oracle_lib, files)
    assert accepted > 50 and rejected > 50, (accepted, rejected)


def test_seeded_mutations_verdicts_match_the_parser(cuda_ready, oracle_lib):
    """Byte flips in the index and payloads (and a few in the header) of valid files of both
    types and every tile shape."""
    rng = np.random.default_rng(4242)
    bases = []
    for k, (kind, w, h, tile) in enumerate([("u16", 150, 90, (64, 64)), ("f32", 140, 70, (128, 32)),
                                             ("u16", 300, 40, (256, 16)), ("u16", 65, 33, (128, 32)),
                                             ("f32", 64, 64, (64, 64))]):
        img = (workloads.detector_frame(w, h, seed=900 + k) if kind == "u16"
               else workloads.field_frame(w, h, seed=900 + k))
        bases.append(oracle_lib.compress_image(img, tile))
    files = []
    for i in range(1200):
        b = bytearray(bases[i % len(bases)])
        for _ in range(int(rng.integers(1, 4))):
            lo = 0 if rng.random() < 0.05 else 64
            pos = int(rng.integers(lo, len(b)))
            b[pos] ^= int(rng.integers(1, 256))
        files.append(bytes(b))
    accepted, rejected = verdicts(oracle_lib, files)
    assert rejected > 100 and accepted > 10, (accepted, rejected)


def test_header_must_match_the_host_copy(cuda_ready, oracle_lib):
    img = workloads.detector_frame(200, 100, seed=5)
    file = oracle_lib.compress_image(img, (64, 64))
    b = Batch([file])
    # The device bytes differ from the checked header in a field the host does not read back.
    other = bytearray(file)
    other[30] ^= 1  # reserved header bytes: the host copy is clean, the device copy is not
    src = to_device(np.frombuffer(bytes(other), np.uint8))
    b.keep.append(src)
    b.entries[0] = (ConstBytes(src.data_ptr(), len(file)), file[:64], b.entries[0][2])
    assert b.run() == Status.success
    assert b.records()[0] == (int(Status.malformed_data), 0)


def test_host_argument_checks(cuda_ready, oracle_lib):
    img = workloads.detector_frame(100, 60, seed=6)
    file = oracle_lib.compress_image(img, (128, 32))
    b = Batch([file])
    res = ResultBuffer(b.results.data_ptr(), 1)
    src, head, view = b.entries[0]
    call = cuda.decode_unparsed_async
    assert call([], res) == Status.success
    assert call([(src, head, view)] * 17, ResultBuffer(b.results.data_ptr(), 17)) == \
        Status.resource_limit
    assert call([(src, head, view)], ResultBuffer(b.results.data_ptr(), 0)) == \
        Status.buffer_too_small
    assert call([(src, head, view)], ResultBuffer(0, 1)) == Status.invalid_argument
    assert call([(ConstBytes(src.data + 2, len(file)), head, view)], res) == \
        Status.invalid_argument  # misaligned file
    assert call([(ConstBytes(src.data, len(file) - 4), head, view)], res) == \
        Status.malformed_data  # the header's file size disagrees
    wrong = api.ImageView(view.data, api.image_spec(2, 100, 60), view.pitch_bytes * 2,
                          view.capacity_bytes * 2)
    assert call([(src, head, wrong)], res) == Status.invalid_argument  # not the file's type
    alias = api.ImageView(src.data, view.image, view.pitch_bytes, view.capacity_bytes)
    assert call([(src, head, alias)], res) == Status.invalid_argument  # output over the input
    assert call([(src, head, view), (src, head, view)], ResultBuffer(b.results.data_ptr(), 2)) \
        == Status.invalid_argument  # two outputs in one place
    bad = bytearray(file[:64])
    bad[8] = 9  # version
    assert call([(src, bytes(bad), view)], res) == Status.unsupported_format
    assert b.run() == Status.success and b.records()[0][0] == 0
