"""TEST INFRASTRUCTURE ONLY: ctypes access to the CPU oracle and to the reference CPU codec.

`Oracle` wraps oracle/liboracle.so, the plain-C restatement of the reference CPU codec
(tsc_oracle.c) plus the seeded case generators (oracle_cases.cpp). `Reference` wraps
oracle/_ref/libtsref.so, the reference's own CPU codec compiled from its sources by
oracle/Makefile (present only where the reference checkout was available at build time).

Only tests/, __graft_entry__.smoke() and bench.py (cpu_baseline and --impl reference) import this
module. The product library never loads either shared object.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libtsref.so")

def reference_dir() -> str | None:
    """The reference checkout named by the TILESTREAM_REFERENCE environment variable, when that
    names a directory; None otherwise (no path is assumed)."""
    path = os.environ.get("TILESTREAM_REFERENCE")
    return path if path and os.path.isdir(path) else None


UINT16, FLOAT32 = 1, 2
RAW, CONSTANT, PREDICT = 0, 1, 2
SAMPLE = {UINT16: 2, FLOAT32: 4}
DTYPE = {UINT16: np.uint16, FLOAT32: np.uint32}

# Allocation budgets of the reference fuzz harness (fuzz/harness.h:24).
FUZZ_LIMITS = (1 << 20, 1 << 15, 8 << 20)

TILE_DTYPE = np.dtype([("mode", "<u4"), ("width", "<u2"), ("height", "<u2"), ("offset", "<u8"),
                       ("length", "<u8"), ("first_segment", "<u8")])
SEGMENT_DTYPE = np.dtype([("seed", "<u4"), ("bit_width", "<u4"), ("payload_offset", "<u8"),
                          ("payload_bytes", "<u8")])


class Layout(C.Structure):
    _fields_ = [("type", C.c_uint32), ("width", C.c_uint32), ("height", C.c_uint32),
                ("tile_width", C.c_uint16), ("tile_height", C.c_uint16),
                ("file_bytes", C.c_uint64), ("tile_count", C.c_uint64),
                ("segment_count", C.c_uint64)]


class Limits(C.Structure):
    _fields_ = [("file_bytes", C.c_uint64), ("tile_count", C.c_uint64),
                ("metadata_bytes", C.c_uint64)]


def build(reference: bool = True) -> None:
    """Compiles liboracle.so, and oracle/_ref when TILESTREAM_REFERENCE names the reference
    checkout (an already built oracle/_ref is kept otherwise)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    ref = reference_dir()
    if reference and ref and os.path.isdir(os.path.join(ref, "src", "cpu")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref}"], check=True)


def _ptr(a) -> C.c_void_p:
    if a is None:
        return C.c_void_p(0)
    if isinstance(a, (bytes, bytearray)):
        a = np.frombuffer(a, dtype=np.uint8)
    return C.c_void_p(a.ctypes.data)


def as_bytes(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a).view(np.uint8).reshape(-1)


class Oracle:
    """The C oracle. Methods mirror the reference CPU API with numpy buffers."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build(reference=False)
        lib = C.CDLL(path)
        u32, u64, vp = C.c_uint32, C.c_uint64, C.c_void_p
        lib.tso_compress_bound.argtypes = [u32, u32, u32, u32, u32, C.POINTER(u64)]
        lib.tso_image_span.argtypes = [u32, u32, u32, u64, C.POINTER(u64)]
        lib.tso_compress.argtypes = [vp, u32, u32, u32, u64, u64, u32, u32, vp, u64,
                                     C.POINTER(u64)]
        lib.tso_decompress.argtypes = [vp, u64, vp, u32, u32, u32, u64, u64, C.POINTER(Limits)]
        lib.tso_parse_layout.argtypes = [vp, u64, C.POINTER(Limits), C.POINTER(Layout)]
        lib.tso_parse_fill.argtypes = [vp, u64, C.POINTER(Layout), vp, vp]
        lib.tso_calibrate.argtypes = [C.c_float, C.c_float, C.c_float]
        lib.tso_calibrate.restype = C.c_float
        lib.tso_calibrate_f64.argtypes = [C.c_float, C.c_float, C.c_float]
        lib.tso_calibrate_f64.restype = C.c_double
        lib.tso_calibrate_image.argtypes = [vp, u32, u32, u32, u64, C.c_float, vp, u64,
                                            C.c_float, vp, u64, vp, u64]
        lib.tso_case.argtypes = [u64, C.POINTER(u32), C.POINTER(u64), vp]
        lib.tso_fill.argtypes = [u32, u32, u32, u64, u32, u64, vp]
        lib.tso_mutation_build.argtypes = [vp, u64, vp, u64, C.POINTER(u64)]
        lib.tso_rng_new.argtypes = [u64]
        lib.tso_rng_new.restype = vp
        lib.tso_rng_free.argtypes = [vp]
        lib.tso_rng_next.argtypes = [vp]
        lib.tso_rng_next.restype = u64
        lib.tso_fabricate.argtypes = [vp, vp, C.POINTER(u64), vp, C.POINTER(u64), C.POINTER(u64)]
        self.lib = lib

    # --- sizes -----------------------------------------------------------------------------
    def compress_bound(self, ptype, width, height, tile=(128, 32)):
        out = C.c_uint64(0)
        st = self.lib.tso_compress_bound(ptype, width, height, tile[0], tile[1], C.byref(out))
        return st, out.value

    def image_span(self, ptype, width, height, pitch):
        out = C.c_uint64(0)
        st = self.lib.tso_image_span(ptype, width, height, pitch, C.byref(out))
        return st, out.value

    # --- codec -----------------------------------------------------------------------------
    def compress(self, pixels: np.ndarray, ptype: int, width: int, height: int, pitch: int,
                 tile=(128, 32)) -> bytes:
        """Encodes a pitched image given as a flat byte array; returns the .tsc file."""
        buf = as_bytes(pixels)
        st, bound = self.compress_bound(ptype, width, height, tile)
        if st:
            raise ValueError(f"compress_bound status {st}")
        out = np.zeros(bound, dtype=np.uint8)
        written = C.c_uint64(0)
        st = self.lib.tso_compress(_ptr(buf), ptype, width, height, pitch, buf.size, tile[0],
                                   tile[1], _ptr(out), bound, C.byref(written))
        if st:
            raise ValueError(f"oracle compress status {st}")
        return out[:written.value].tobytes()

    def compress_image(self, image: np.ndarray, tile=(128, 32)) -> bytes:
        ptype = UINT16 if image.dtype == np.uint16 else FLOAT32
        image = np.ascontiguousarray(image)
        h, w = image.shape
        return self.compress(image, ptype, w, h, w * SAMPLE[ptype], tile)

    def decompress(self, file: bytes, ptype: int, width: int, height: int, pitch: int | None = None,
                   limits=None, fill: int = 0):
        """Returns (status, flat byte buffer of pitch * height)."""
        s = SAMPLE.get(ptype, 2)
        pitch = pitch if pitch is not None else width * s
        out = np.full(pitch * height, fill, dtype=np.uint8)
        src = np.frombuffer(file, dtype=np.uint8) if len(file) else np.zeros(1, np.uint8)
        lim = C.byref(Limits(*limits)) if limits is not None else None
        st = self.lib.tso_decompress(_ptr(src), len(file), _ptr(out), ptype, width, height, pitch,
                                     out.size, lim)
        return st, out

    def decompress_image(self, file: bytes) -> np.ndarray:
        st, meta = self.parse(file)
        if st:
            raise ValueError(f"oracle parse status {st}")
        ptype, w, h = meta["type"], meta["width"], meta["height"]
        st, out = self.decompress(file, ptype, w, h)
        if st:
            raise ValueError(f"oracle decompress status {st}")
        return out.view(DTYPE[ptype]).reshape(h, w)

    def parse(self, file: bytes, limits=None):
        """Returns (status, metadata dict with numpy tile and segment tables)."""
        src = np.frombuffer(file, dtype=np.uint8) if len(file) else np.zeros(1, np.uint8)
        lay = Layout()
        lim = C.byref(Limits(*limits)) if limits is not None else None
        st = self.lib.tso_parse_layout(_ptr(src), len(file), lim, C.byref(lay))
        if st:
            return st, None
        tiles = np.zeros(lay.tile_count, dtype=TILE_DTYPE)
        segs = np.zeros(max(lay.segment_count, 1), dtype=SEGMENT_DTYPE)
        st = self.lib.tso_parse_fill(_ptr(src), len(file), C.byref(lay), _ptr(tiles), _ptr(segs))
        if st:
            return st, None
        return 0, {"type": lay.type, "width": lay.width, "height": lay.height,
                   "tile": (lay.tile_width, lay.tile_height), "file_bytes": lay.file_bytes,
                   "tiles": tiles, "segments": segs[:lay.segment_count]}

    # --- calibration ------------------------------------------------------------------------
    def calibrate(self, x: float, offset: float, gain: float) -> float:
        return self.lib.tso_calibrate(x, offset, gain)

    def calibrate_f64(self, x: float, offset: float, gain: float) -> float:
        return self.lib.tso_calibrate_f64(x, offset, gain)

    def calibrate_image(self, samples: np.ndarray, offset, gain) -> np.ndarray:
        """samples: (h, w) uint16 or uint32 (FP32 words); offset/gain: float or (h, w) float32."""
        samples = np.ascontiguousarray(samples)
        h, w = samples.shape
        ptype = UINT16 if samples.dtype == np.uint16 else FLOAT32
        out = np.empty((h, w), dtype=np.float32)
        om = np.ascontiguousarray(offset, dtype=np.float32) if np.ndim(offset) else None
        gm = np.ascontiguousarray(gain, dtype=np.float32) if np.ndim(gain) else None
        self.lib.tso_calibrate_image(
            _ptr(samples), ptype, w, h, w * SAMPLE[ptype],
            0.0 if om is not None else float(offset), _ptr(om), w * 4,
            1.0 if gm is not None else float(gain), _ptr(gm), w * 4, _ptr(out), w * 4)
        return out

    # --- seeded cases -----------------------------------------------------------------------
    def case(self, seed: int) -> dict:
        """The reference robustness case of this seed (tests/robustness/cases.h:147-170)."""
        info = (C.c_uint32 * 10)()
        pitch = C.c_uint64(0)
        self.lib.tso_case(seed, info, C.byref(pitch), None)
        buf = np.empty(pitch.value * info[2], dtype=np.uint8)
        self.lib.tso_case(seed, info, C.byref(pitch), _ptr(buf))
        return {"seed": seed, "type": info[0], "width": info[1], "height": info[2],
                "tile": (info[3], info[4]), "pattern": info[5],
                "roi": (info[6], info[7], info[8], info[9]), "pitch": pitch.value, "bytes": buf}

    def fill(self, ptype, width, height, pattern, seed, pitch=None) -> np.ndarray:
        pitch = pitch or width * SAMPLE[ptype]
        buf = np.zeros(pitch * height, dtype=np.uint8)
        self.lib.tso_fill(ptype, width, height, pitch, pattern, seed, _ptr(buf))
        return buf

    def engine(self, seed: int) -> "Engine":
        """A std::mt19937_64 engine shared by Python draws and fabricate()."""
        return Engine(self.lib, seed)

    def fabricate(self, engine: "Engine", tiles: np.ndarray, segments: np.ndarray,
                  file_bytes: int):
        """One fabricated change of parsed metadata (tests/cuda_robustness_test.cpp:194-243):
        returns (tiles, segments, file_bytes) copies with one field changed or one record
        dropped. tiles/segments use TILE_DTYPE/SEGMENT_DTYPE."""
        t = np.ascontiguousarray(tiles.copy())
        g = np.zeros(len(segments) + 1, SEGMENT_DTYPE)
        g[:len(segments)] = segments
        nt, ng, fb = C.c_uint64(len(t)), C.c_uint64(len(segments)), C.c_uint64(file_bytes)
        self.lib.tso_fabricate(engine.handle, _ptr(t), C.byref(nt), _ptr(g), C.byref(ng),
                               C.byref(fb))
        return t[:nt.value].copy(), g[:ng.value].copy(), fb.value

    def mutation_file(self, corpus_input: bytes):
        """Rebuilds the mutated .tsc file of one reference mutation-corpus input, or None."""
        cap = 1 << 22
        out = np.zeros(cap, dtype=np.uint8)
        size = C.c_uint64(0)
        src = np.frombuffer(corpus_input, dtype=np.uint8) if corpus_input else np.zeros(1, np.uint8)
        rc = self.lib.tso_mutation_build(_ptr(src), len(corpus_input), _ptr(out), cap,
                                         C.byref(size))
        return None if rc else out[:size.value].tobytes()


class Engine:
    """std::mt19937_64 in the oracle library; next() is one engine draw."""

    def __init__(self, lib, seed: int):
        self.lib = lib
        self.handle = lib.tso_rng_new(seed)

    def next(self) -> int:
        return int(self.lib.tso_rng_next(self.handle))

    def __del__(self):
        if getattr(self, "handle", None):
            self.lib.tso_rng_free(self.handle)
            self.handle = None


class Reference:
    """The reference CPU codec itself (oracle/_ref/libtsref.so), when it was built."""

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_SO)

    def __init__(self, path: str = REF_SO):
        lib = C.CDLL(path)
        u32, u64, vp = C.c_uint32, C.c_uint64, C.c_void_p
        lib.tsr_compress_bound.argtypes = [u32, u32, u32, u32, u32, C.POINTER(u64)]
        lib.tsr_image_span.argtypes = [u32, u32, u32, u64, C.POINTER(u64)]
        lib.tsr_workspace_size.argtypes = [u64, u64, u32, u32, u64, C.POINTER(u64)]
        lib.tsr_compress.argtypes = [vp, u32, u32, u32, u64, u64, u32, u32, vp, u64,
                                     C.POINTER(u64)]
        lib.tsr_decompress.argtypes = [vp, u64, vp, u32, u32, u32, u64, u64, vp]
        lib.tsr_parse.argtypes = [vp, u64, vp, vp, vp, u64, vp, u64]
        self.lib = lib

    def compress_bound(self, ptype, width, height, tile=(128, 32)):
        out = C.c_uint64(0)
        st = self.lib.tsr_compress_bound(ptype, width, height, tile[0], tile[1], C.byref(out))
        return st, out.value

    def image_span(self, ptype, width, height, pitch):
        out = C.c_uint64(0)
        st = self.lib.tsr_image_span(ptype, width, height, pitch, C.byref(out))
        return st, out.value

    def workspace_size(self, images, tiles, tile, temp):
        out = C.c_uint64(0)
        st = self.lib.tsr_workspace_size(images, tiles, tile[0], tile[1], temp, C.byref(out))
        return st, out.value

    def compress(self, pixels, ptype, width, height, pitch, tile=(128, 32)) -> bytes:
        buf = as_bytes(pixels)
        st, bound = self.compress_bound(ptype, width, height, tile)
        if st:
            raise ValueError(f"compress_bound status {st}")
        out = np.zeros(bound, dtype=np.uint8)
        written = C.c_uint64(0)
        st = self.lib.tsr_compress(_ptr(buf), ptype, width, height, pitch, buf.size, tile[0],
                                   tile[1], _ptr(out), bound, C.byref(written))
        if st:
            raise ValueError(f"reference compress status {st}")
        return out[:written.value].tobytes()

    def compress_image(self, image: np.ndarray, tile=(128, 32)) -> bytes:
        ptype = UINT16 if image.dtype == np.uint16 else FLOAT32
        image = np.ascontiguousarray(image)
        h, w = image.shape
        return self.compress(image, ptype, w, h, w * SAMPLE[ptype], tile)

    def decompress(self, file: bytes, ptype, width, height, pitch=None, limits=None, fill=0,
                   out=None):
        s = SAMPLE.get(ptype, 2)
        pitch = pitch if pitch is not None else width * s
        if out is None:
            out = np.full(pitch * height, fill, dtype=np.uint8)
        src = np.frombuffer(file, dtype=np.uint8) if len(file) else np.zeros(1, np.uint8)
        lim = np.array(limits, dtype=np.uint64) if limits is not None else None
        st = self.lib.tsr_decompress(_ptr(src), len(file), _ptr(out), ptype, width, height,
                                     pitch, out.size, _ptr(lim))
        return st, out

    def parse_status(self, file: bytes) -> int:
        """One reference parse_metadata call (its tables are built, not copied out)."""
        src = np.frombuffer(file, dtype=np.uint8) if len(file) else np.zeros(1, np.uint8)
        info = np.zeros(8, dtype=np.uint64)
        return self.lib.tsr_parse(_ptr(src), len(file), None, _ptr(info), None, 0, None, 0)

    def parse(self, file: bytes, limits=None):
        src = np.frombuffer(file, dtype=np.uint8) if len(file) else np.zeros(1, np.uint8)
        lim = np.array(limits, dtype=np.uint64) if limits is not None else None
        info = np.zeros(8, dtype=np.uint64)
        st = self.lib.tsr_parse(_ptr(src), len(file), _ptr(lim), _ptr(info), None, 0, None, 0)
        if st:
            return st, None
        tiles = np.zeros(int(info[6]), dtype=TILE_DTYPE)
        segs = np.zeros(max(int(info[7]), 1), dtype=SEGMENT_DTYPE)
        self.lib.tsr_parse(_ptr(src), len(file), _ptr(lim), _ptr(info), _ptr(tiles), tiles.size,
                           _ptr(segs), segs.size)
        return 0, {"type": int(info[0]), "width": int(info[1]), "height": int(info[2]),
                   "tile": (int(info[3]), int(info[4])), "file_bytes": int(info[5]),
                   "tiles": tiles, "segments": segs[:int(info[7])]}
