"""The reference's own C++ callers of the drop-in API, compiled unchanged against include/ and
this library by tests/reference_suite/Makefile (from the reference checkout, at build time):

* its CUDA test suites tests/cuda_{api,loading,encoder,decoder,calibration,numerics,robustness}
  _test.cpp with tests/cuda_test_main.cpp, on a GoogleTest-compatible harness of this
  repository (tests/reference_suite/gtest/gtest.h) and the static library (one executable, one
  CUDA runtime, as in the reference build). These hold the API contract tests: independent
  plans on two streams and two host threads, memory returned after repeated cycles, no hidden
  device synchronization, enqueue is not completion, DeviceBuffer ownership, a caller's pending
  error blocks enqueue (cuda_api_test.cpp:209-365), first executions that do not wait on a held
  stream (cuda_loading_test.cpp:130-160), and the codec, validation, calibration contract and
  robustness suites;
* tests/cuda_headers_test.cu, the compile-time signature and layout asserts;
* examples/cpp_client/main.cpp, linked with the shared libtilestream_b200.so.

The binaries travel with the repository (they are built artefacts, not committed); these tests
check that they were linked against the current library build.
"""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SUITE_DIR = os.path.join(HERE, "reference_suite")
BIN = os.path.join(SUITE_DIR, "_ref")
SUITES = ("api", "loading", "encoder", "decoder", "calibration", "numerics", "robustness")


def _library_stamp():
    with open(os.path.join(ROOT, "tilestream_b200", "_build", "stamp")) as f:
        return f.read().strip()


def _binary(name):
    path = os.path.join(BIN, name)
    if not os.path.exists(path):
        import oracle
        if oracle.reference_dir() is None:
            pytest.skip("reference callers not built (set TILESTREAM_REFERENCE and build)")
        subprocess.run(["make", "-s", "-C", SUITE_DIR], check=True)
    stamp = os.path.join(BIN, "stamp")
    assert os.path.exists(stamp), "reference callers have no library stamp"
    with open(stamp) as f:
        assert f.read().strip() == _library_stamp(), \
            "reference callers were linked against an older library build: rebuild them"
    return path


def _run(args, timeout):
    r = subprocess.run(args, capture_output=True, text=True, timeout=timeout)
    return r.returncode, r.stdout + r.stderr


def test_reference_header_asserts():
    """tests/cuda_headers_test.cu compiles against include/ (static_asserts on the five executor
    signatures, BatchPlan move/copy traits, record layouts) and runs."""
    import oracle
    if oracle.reference_dir() is not None:
        subprocess.run(["make", "-s", "-C", SUITE_DIR, "_ref/tilestream_cuda_header_tests"],
                       check=True)
    rc, out = _run([_binary("tilestream_cuda_header_tests")], 60)
    assert rc == 0, out


@pytest.mark.gpu
@pytest.mark.parametrize("suite", SUITES)
def test_reference_cuda_suite(cuda_ready, suite):
    rc, out = _run([_binary(f"tilestream_cuda_{suite}_tests")], 1200)
    tail = "\n".join(out.splitlines()[-40:])
    assert rc == 0, tail
    assert "[==========]" in out and " 0 failed" in out, tail


@pytest.mark.gpu
def test_reference_cpp_client(cuda_ready):
    """examples/cpp_client/main.cpp: CPU round trips, then GPU encode -> trusted decode -> fused
    dark-frame calibration of three frames, each checked bit for bit by the client."""
    rc, out = _run([_binary("cpp_client")], 300)
    assert rc == 0, out
    assert "GPU frame 2" in out, out
