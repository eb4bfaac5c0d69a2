"""The library's binary interface, checked without a GPU: libtilestream_b200.so loads, exports
every C entry point that include/tilestream_c.h declares and every free function and member
that the drop-in C++ headers declare, the Python bindings cover the C header exactly, and
every ctypes record has the layout gcc gives the C record."""
import ctypes
import os
import re
import subprocess
import tempfile

import pytest

from tilestream_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
C_HEADER = os.path.join(ROOT, "include", "tilestream_c.h")

# Free functions and members of the C++ headers (header:line of each declaration).
CXX_SYMBOLS = [
    "tilestream::image_span(",                     # sizing.h:28
    "tilestream::compress_bound(",                 # sizing.h:30
    "tilestream::workspace_size(",                 # sizing.h:32
    "tilestream::parse_metadata(",                 # api.h:44
    "tilestream::cpu::compress(",                  # cpu.h:9
    "tilestream::cpu::decompress(",                # cpu.h:11
    "tilestream::version()",                       # info.h:7
    "tilestream::info_json[abi:cxx11]()",          # info.h:8
    "tilestream::cuda::synchronize(",              # cuda.h:152
    "tilestream::cuda::prepare_batch(",            # cuda.h:184
    "tilestream::cuda::compress_async(",           # cuda.h:186
    "tilestream::cuda::decompress_async(",         # cuda.h:188
    "tilestream::cuda::decode_roi_async(",         # cuda.h:190
    "tilestream::cuda::calibrate_async(",          # cuda.h:192
    "tilestream::cuda::decode_calibrate_async(",   # cuda.h:194
    "tilestream::cuda::DeviceBuffer::allocate(",   # cuda.h:131
    "tilestream::cuda::DeviceBuffer::release(",    # cuda.h:134
    "tilestream::cuda::DeviceBuffer::~DeviceBuffer()",
    "tilestream::cuda::BatchPlan::workspace_spec() const",  # cuda.h:163
    "tilestream::cuda::BatchPlan::~BatchPlan()",
    "tilestream::cuda::prepare_mixed_batch(",      # batch.h:57
    "tilestream::cuda::run_mixed_batch(",          # batch.h:62
    "tilestream::cuda::mixed_batch_stats(",        # batch.h:63
    "tilestream::cuda::Server::create(",           # serve.h:75
    "tilestream::cuda::Server::add_archive(",      # serve.h:79
    "tilestream::cuda::Server::seal()",            # serve.h:82
    "tilestream::cuda::Server::run(",              # serve.h:86
    "tilestream::cuda::Server::pool() const",      # serve.h:89
    "tilestream::cuda::roi_staging_size(",         # staging.h:23
    "tilestream::cuda::stage_roi_tiles(",          # staging.h:35
]


def c_declarations():
    text = open(C_HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    functions = sorted(set(re.findall(r"\b(ts_\w+)\s*\(", text)))
    records = sorted(set(re.findall(r"}\s*(ts_\w+)\s*;", text)))
    return functions, records


@pytest.fixture(scope="module")
def library():
    return N.lib()


@pytest.fixture(scope="module")
def exported():
    out = subprocess.run(["nm", "-DC", "--defined-only", N.library_path()], check=True,
                         capture_output=True, text=True).stdout
    return out


def test_every_c_entry_point_is_exported(library, exported):
    functions, _ = c_declarations()
    assert len(functions) >= 36
    defined = {line.split()[-1] for line in exported.splitlines() if " T " in line}
    for name in functions:
        assert name in defined, name
        assert getattr(library, name) is not None


def test_bindings_cover_the_header():
    functions, _ = c_declarations()
    assert sorted(N._SIGNATURES) == functions


def test_cxx_api_is_exported(exported):
    text = " ".join(line.split(" ", 2)[-1] for line in exported.splitlines()
                    if " T " in line or " W " in line)
    for symbol in CXX_SYMBOLS:
        assert symbol in text, symbol


def camel(name):
    return "".join(part.capitalize() for part in name[3:].split("_"))


def test_record_layouts_match_gcc():
    _, records = c_declarations()
    assert "ts_serve_outcome" in records and "ts_batch_item" in records
    src = ['#include <stdio.h>', '#include <stddef.h>', '#include "tilestream_c.h"',
           "int main(void) {"]
    for r in records:
        src.append(f'printf("{r} %zu %zu\\n", sizeof({r}), _Alignof({r}));')
        for field, _ in getattr(N, camel(r))._fields_:
            src.append(f'printf("{r}.{field} %zu\\n", offsetof({r}, {field}));')
    src.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "layout.c")
        exe = os.path.join(d, "layout")
        with open(c, "w") as f:
            f.write("\n".join(src))
        subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), c, "-o", exe],
                       check=True)
        lines = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    for line in lines.splitlines():
        parts = line.split()
        if "." in parts[0]:
            rec, field = parts[0].split(".")
            cls = getattr(N, camel(rec))
            assert getattr(cls, field).offset == int(parts[1]), parts[0]
        else:
            cls = getattr(N, camel(parts[0]))
            assert ctypes.sizeof(cls) == int(parts[1]), parts[0]
            assert ctypes.alignment(cls) == int(parts[2]), parts[0]
