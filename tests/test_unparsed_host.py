"""The host half of decode_unparsed_async, with stand-in device addresses: argument checks, and
the header check's statuses against parse_metadata's on every file of the reference's fuzz
corpora. A file whose header passes goes on to the device checks, which fail on stand-in
addresses (cuda_error without a GPU, invalid_argument with one: not device memory); every other
call must return parse_metadata's own status, before any device call."""
import struct

import numpy as np
import pytest

from tilestream_b200 import api, cuda
from tilestream_b200.api import ConstBytes, ResultBuffer, Status

FAKE_FILE = 1 << 40      # stand-in device addresses: never dereferenced by the host checks
FAKE_OUT = 1 << 41
FAKE_RESULTS = 1 << 42
# What a call returns once the header has passed and the device checks meet the stand-ins.
PASSED = (Status.cuda_error, Status.invalid_argument)


def entry(file: bytes, size=None, out=None):
    ptype, width, height = 1, 1, 1
    if len(file) >= 64:
        ptype = file[14] if file[14] in (1, 2) else 1
        width, height = struct.unpack_from("<II", file, 16)
        width, height = max(width, 1), max(height, 1)
    s = 4 if ptype == 2 else 2
    pitch = (width * s + 15) // 16 * 16
    view = out or api.ImageView(FAKE_OUT, api.image_spec(ptype, width, height), pitch,
                                pitch * height)
    return (ConstBytes(FAKE_FILE, len(file) if size is None else size), file[:64], view)


def call(entries, count=None):
    n = len(entries) if count is None else count
    return cuda.decode_unparsed_async(entries, ResultBuffer(FAKE_RESULTS, n))


def test_header_statuses_match_the_parser():
    from golden import inputs
    checked = passed = 0
    for name, data in inputs.corpus("parse"):
        if len(data) == 0:
            continue
        st_parse, _ = api.parse_metadata(np.frombuffer(data, np.uint8), size=len(data))
        st = call([entry(data)])
        if st in PASSED and st_parse not in PASSED:
            passed += 1  # the header passed; the device half cannot run here
            continue
        # Rejected on the host: by the header check, with the parser's status (an output
        # built from a rejected header may also be refused, but only after the header check).
        assert st == st_parse, (name, st, st_parse)
        checked += 1
    assert checked > 20 and passed > 20, (checked, passed)


def test_argument_checks():
    file = bytes(64)
    e = entry(file)
    assert call([]) == Status.success
    assert cuda.decode_unparsed_async([e], ResultBuffer(0, 1)) == Status.invalid_argument
    assert call([e] * 17) == Status.resource_limit
    assert call([e], count=0) == Status.buffer_too_small
    assert cuda.decode_unparsed_async([e], ResultBuffer(FAKE_RESULTS + 4, 1)) == \
        Status.invalid_argument  # misaligned records
    assert call([(ConstBytes(FAKE_FILE + 2, 64), file, e[2])]) == Status.invalid_argument
    # A file smaller than a header is malformed, as for parse_metadata.
    assert call([(ConstBytes(FAKE_FILE, 10), file, e[2])]) == Status.malformed_data
    # The result records may not overlap a file.
    assert cuda.decode_unparsed_async([(ConstBytes(FAKE_RESULTS, 64), file, e[2])],
                                      ResultBuffer(FAKE_RESULTS, 1)) == Status.invalid_argument


@pytest.mark.parametrize("field,value,status", [
    (0, 0x00, Status.malformed_data),          # magic
    (8, 2, Status.unsupported_format),         # major version
    (14, 7, Status.unsupported_type),          # pixel type
    (24, 100, Status.unsupported_format),      # tile width
])
def test_header_fields(oracle_lib, field, value, status):
    from tilestream_b200 import workloads
    file = bytearray(oracle_lib.compress_image(workloads.detector_frame(70, 40, seed=8),
                                               (64, 64)))
    assert call([entry(bytes(file))]) in PASSED  # valid header: the device checks are next
    file[field] = value
    assert api.parse_metadata(np.frombuffer(bytes(file), np.uint8))[0] == status
    assert call([entry(bytes(file))]) == status
