"""Regenerates the golden .tsc fixtures of this directory with the reference's own encoder.

The eight single-tile cases are the hand-calculated golden inputs of the reference tests
(tests/cpu_codec_test.cpp:86-104 for uint16, tests/fp32_codec_test.cpp:81-82 for float32). Each
input is encoded by the reference CPU codec compiled from its sources (oracle/_ref, built by
oracle/Makefile) and written as a .hex file in the reference's text layout. When the reference
checkout is present the script also asserts that every regenerated file equals the reference's
own golden file byte for byte.

It also records the C1 golden round trip (uint16 1024x1024 frame, seed 1, tiles 128x32): the
SHA-256 and size of the reference encoding, in c1_roundtrip.json.

And it extracts the reference's calibration contract rows (tests/numerics/support.h:404-456:
special-value inputs with their exact expected words, which the reference runs through its host
form and every GPU calibration path, tests/numerics_test.cpp:79-87,
tests/cuda_numerics_test.cpp:161-200) into calibration_contract_rows.json, after checking that
the oracle's host form reproduces each of them.

And it copies the reference's committed test inputs that the GPU parity tests replay, so that
no test needs the reference checkout at run time: the two fuzz corpora (fuzz/corpus/parse and
fuzz/corpus/mutation, every file) into fuzz_corpus.npz, and the four image fixtures
(datasets/fixtures/*.npy) into datasets/.

Run from the repository root, with TILESTREAM_REFERENCE naming the reference checkout:
    TILESTREAM_REFERENCE=<checkout> python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import re
import shutil
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from tilestream_b200 import workloads  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def cases():
    zero_width = [0x0102] * 8 + [0x0304] * 8
    half_range = [0, 32768, 0, 32768, 0, 32768, 0, 32768, 0] + [5] * 9
    u16 = np.uint16
    return [
        ("uint16_raw", 1, 1, np.array([0x1234], u16), oracle.RAW),
        ("uint16_constant", 3, 2, np.full(6, 0xbeef, u16), oracle.CONSTANT),
        ("uint16_wrap", 8, 2, np.array([65535, 0, 1, 2, 3, 4, 5, 6, 0, 65535, 65534, 65533,
                                        65532, 65531, 65530, 65529], u16), oracle.PREDICT),
        ("uint16_zero_width", 8, 2, np.array(zero_width, u16), oracle.PREDICT),
        ("uint16_raw_tie", 6, 1, np.arange(6, dtype=u16), oracle.RAW),
        ("uint16_half_range", 9, 2, np.array(half_range, u16), oracle.PREDICT),
        ("float32_raw", 1, 1, np.array([0x7fc01234], np.uint32), oracle.RAW),
        ("float32_negative_zero_constant", 3, 2, np.full(6, 0x80000000, np.uint32),
         oracle.CONSTANT),
    ]


def to_hex(data: bytes) -> str:
    """Eight bytes per line for the 64-byte header and each 32-byte index entry, then the
    payload, as in the reference's golden files."""
    lines = [" ".join(f"{b:02x}" for b in data[i:i + 8]) for i in range(0, len(data), 8)]
    return "\n".join(lines) + "\n"


def read_hex(path: str) -> bytes:
    with open(path) as f:
        return bytes(int(tok, 16) for tok in f.read().split())


def reference_checkout() -> str:
    ref = oracle.reference_dir()
    if ref is None:
        raise SystemExit("set TILESTREAM_REFERENCE to the reference checkout")
    return ref


def copy_reference_inputs(ref: str) -> None:
    """fuzz_corpus.npz (key '<corpus>/<file name>', the file's bytes) and datasets/*.npy."""
    corpus = {}
    for kind in ("parse", "mutation"):
        folder = os.path.join(ref, "fuzz", "corpus", kind)
        for name in sorted(os.listdir(folder)):
            with open(os.path.join(folder, name), "rb") as f:
                corpus[f"{kind}/{name}"] = np.frombuffer(f.read(), np.uint8)
    np.savez_compressed(os.path.join(HERE, "fuzz_corpus.npz"), **corpus)
    out = os.path.join(HERE, "datasets")
    os.makedirs(out, exist_ok=True)
    folder = os.path.join(ref, "datasets", "fixtures")
    for name in sorted(os.listdir(folder)):
        if name.endswith(".npy"):
            shutil.copyfile(os.path.join(folder, name), os.path.join(out, name))


def contract_rows():
    """The rows of the reference's contract_rows[] table, read from its header text."""
    with open(os.path.join(reference_checkout(), "tests", "numerics", "support.h")) as f:
        text = f.read()
    block = text[text.index("contract_rows[] = {"):]
    block = block[:block.index("};")]
    word = r"(0x[0-9a-fA-F]{8})"
    rows = re.findall(r"\{" + ", ".join([word] * 4) + r', "([^"]*)"\}', block)
    assert len(rows) == block.count('"') // 2, "a row did not parse"
    return [{"x": x, "offset": o, "gain": g, "expected": e, "note": n}
            for x, o, g, e, n in rows]


def same_word(got: int, want: int) -> bool:
    """Equal words, or both NaN (the contract compares NaNs by class)."""
    nan = lambda w: (w & 0x7f800000) == 0x7f800000 and (w & 0x007fffff) != 0  # noqa: E731
    return got == want or (nan(got) and nan(want))


def main():
    ref_dir = reference_checkout()
    copy_reference_inputs(ref_dir)
    rows = contract_rows()
    words = lambda key: np.array([[int(r[key], 16) for r in rows]], np.uint32)  # noqa: E731
    got = oracle.Oracle().calibrate_image(words("x"), words("offset").view(np.float32),
                                          words("gain").view(np.float32)).view(np.uint32)[0]
    for r, g in zip(rows, got):
        assert same_word(int(g), int(r["expected"], 16)), (r["note"], hex(int(g)))
    with open(os.path.join(HERE, "calibration_contract_rows.json"), "w") as f:
        json.dump(rows, f, indent=1)
        f.write("\n")

    ref = oracle.Reference()
    manifest = {}
    for name, w, h, pixels, mode in cases():
        ptype = oracle.UINT16 if pixels.dtype == np.uint16 else oracle.FLOAT32
        data = ref.compress(pixels, ptype, w, h, w * oracle.SAMPLE[ptype])
        path = os.path.join(HERE, name + ".hex")
        with open(path, "w") as f:
            f.write(to_hex(data))
        manifest[name] = {"width": w, "height": h, "type": ptype, "mode": mode,
                          "pixels": [int(v) for v in pixels]}
        upstream = os.path.join(ref_dir, "tests", "golden", name + ".hex")
        if os.path.exists(upstream):
            assert read_hex(upstream) == data, f"{name}: differs from the reference golden file"
    with open(os.path.join(HERE, "cases.json"), "w") as f:
        json.dump(manifest, f, indent=1)
        f.write("\n")

    frame = workloads.detector_frame(1024, 1024, seed=1)
    data = ref.compress_image(frame, (128, 32))
    st, back = ref.decompress(data, oracle.UINT16, 1024, 1024)
    assert st == 0 and np.array_equal(back.view(np.uint16).reshape(1024, 1024), frame)
    with open(os.path.join(HERE, "c1_roundtrip.json"), "w") as f:
        json.dump({"config": "uint16 1024x1024 detector frame, seed 1, tiles 128x32",
                   "pixels_sha256": hashlib.sha256(frame.tobytes()).hexdigest(),
                   "file_bytes": len(data),
                   "file_sha256": hashlib.sha256(data).hexdigest()}, f, indent=1)
        f.write("\n")
    print("golden fixtures written")


if __name__ == "__main__":
    main()
