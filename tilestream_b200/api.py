"""Python mirror of the reference's public API (include/tilestream/{types,sizing,api}.h).

Names, argument meaning and statuses follow the C++ API; functions return the Status (plus the
value the C++ call writes through a reference) instead of raising, exactly like the reference.
Everything calls libtilestream_b200.so through the C entry points of include/tilestream_c.h.
"""
from __future__ import annotations

import ctypes as C
import enum
import os

import numpy as np

from . import _native as N
from ._native import (BatchItem, BatchRequest, Calibration, CompressedInput, ConstBytes,  # noqa
                      ConstImageView, DeviceResult, ImageSpec, ImageView, MutableBytes,
                      Parameter, ParseLimits, ResultBuffer, Roi, SegmentMetadata, TileMapping,
                      TiffReadLimits, TiffWriteOptions, TileMetadata, TileShape, WorkspaceSpec)


class Status(enum.IntEnum):
    success = 0
    invalid_argument = 1
    invalid_roi = 2
    unsupported_type = 3
    unsupported_format = 4
    malformed_data = 5
    size_overflow = 6
    buffer_too_small = 7
    resource_limit = 8
    cuda_error = 9
    io_error = 10


class PixelType(enum.IntEnum):
    uint16 = 1
    float32 = 2


class TileMode(enum.IntEnum):
    raw = 0
    constant = 1
    predict_bitpack = 2


MAX_BYTES = (1 << 63) - 1
WORKSPACE_ALIGNMENT = 256
TILE_SHAPES = ((128, 32), (64, 64), (256, 16))

TILE_DTYPE = np.dtype([("mode", "<u4"), ("width", "<u2"), ("height", "<u2"), ("offset", "<u8"),
                       ("length", "<u8"), ("first_segment", "<u8")])
SEGMENT_DTYPE = np.dtype([("seed", "<u4"), ("bit_width", "<u4"), ("payload_offset", "<u8"),
                          ("payload_bytes", "<u8")])


def sample_bytes(ptype) -> int:
    return 2 if int(ptype) == PixelType.uint16 else 4


def _ptr(buf) -> int:
    """Address of a numpy array, bytes-like object or torch tensor (0 for None)."""
    if buf is None:
        return 0
    if hasattr(buf, "data_ptr"):
        return int(buf.data_ptr())
    if isinstance(buf, np.ndarray):
        return int(buf.ctypes.data)
    if isinstance(buf, (bytes, bytearray, memoryview)):
        arr = np.frombuffer(buf, dtype=np.uint8)
        return int(arr.ctypes.data) if arr.size else 0
    return int(buf)


def nbytes(buf) -> int:
    if hasattr(buf, "element_size"):
        return int(buf.numel() * buf.element_size())
    if isinstance(buf, np.ndarray):
        return int(buf.nbytes)
    return len(buf)


def const_bytes(buf, size=None) -> ConstBytes:
    return ConstBytes(_ptr(buf), nbytes(buf) if size is None else size)


def mutable_bytes(buf, size=None) -> MutableBytes:
    return MutableBytes(_ptr(buf), nbytes(buf) if size is None else size)


def image_spec(ptype, width, height) -> ImageSpec:
    return ImageSpec(int(ptype), width, height)


def const_view(buf, ptype, width, height, pitch=None, capacity=None) -> ConstImageView:
    pitch = width * sample_bytes(ptype) if pitch is None else pitch
    return ConstImageView(_ptr(buf), image_spec(ptype, width, height), pitch,
                          nbytes(buf) if capacity is None else capacity)


def view(buf, ptype, width, height, pitch=None, capacity=None) -> ImageView:
    pitch = width * sample_bytes(ptype) if pitch is None else pitch
    return ImageView(_ptr(buf), image_spec(ptype, width, height), pitch,
                     nbytes(buf) if capacity is None else capacity)


# --- sizing.h ------------------------------------------------------------------------------

def image_span(image: ImageSpec, pitch_bytes: int):
    out = C.c_uint64(0)
    st = N.lib().ts_image_span(image, pitch_bytes, C.byref(out))
    return Status(st), out.value


def compress_bound(image: ImageSpec, tile: TileShape | None = None):
    out = C.c_uint64(0)
    st = N.lib().ts_compress_bound(image, tile if tile is not None else TileShape(),
                                   C.byref(out))
    return Status(st), out.value


def workspace_size(spec: WorkspaceSpec):
    out = C.c_uint64(0)
    st = N.lib().ts_workspace_size(C.byref(spec), C.byref(out))
    return Status(st), out.value


# --- api.h ---------------------------------------------------------------------------------

class ImageMetadata:
    """An owned tilestream::ImageMetadata, as produced by parse_metadata."""

    def __init__(self, handle: int):
        self.handle = handle

    @classmethod
    def create(cls, image: ImageSpec, tile: TileShape, file_bytes: int, tiles: np.ndarray,
               segments: np.ndarray):
        tiles = np.ascontiguousarray(tiles, dtype=TILE_DTYPE)
        segments = np.ascontiguousarray(segments, dtype=SEGMENT_DTYPE)
        h = C.c_void_p(0)
        st = N.lib().ts_metadata_create(image, tile, file_bytes, _ptr(tiles), tiles.size,
                                        _ptr(segments), segments.size, C.byref(h))
        return Status(st), (cls(h.value) if st == 0 else None)

    def _info(self):
        image, tile = ImageSpec(), TileShape()
        fb, nt, ns = C.c_uint64(), C.c_uint64(), C.c_uint64()
        N.lib().ts_metadata_info(self.handle, C.byref(image), C.byref(tile), C.byref(fb),
                                 C.byref(nt), C.byref(ns))
        return image, tile, fb.value, nt.value, ns.value

    @property
    def image(self) -> ImageSpec:
        return self._info()[0]

    @property
    def tile(self) -> TileShape:
        return self._info()[1]

    @property
    def file_bytes(self) -> int:
        return self._info()[2]

    @property
    def tiles(self) -> np.ndarray:
        n = self._info()[3]
        if n == 0:
            return np.zeros(0, TILE_DTYPE)
        addr = N.lib().ts_metadata_tiles(self.handle)
        return np.frombuffer((C.c_uint8 * (n * 32)).from_address(addr), TILE_DTYPE).copy()

    @property
    def segments(self) -> np.ndarray:
        n = self._info()[4]
        if n == 0:
            return np.zeros(0, SEGMENT_DTYPE)
        addr = N.lib().ts_metadata_segments(self.handle)
        return np.frombuffer((C.c_uint8 * (n * 24)).from_address(addr), SEGMENT_DTYPE).copy()

    def __del__(self, _lib=N.lib):
        # _lib is bound at definition: module globals may already be gone at interpreter exit.
        if getattr(self, "handle", None):
            _lib().ts_metadata_destroy(self.handle)
            self.handle = None


def parse_metadata(source, limits: ParseLimits | None = None, size: int | None = None):
    """Validates a complete host-resident .tsc file; returns (Status, ImageMetadata or None)."""
    h = C.c_void_p(0)
    st = N.lib().ts_parse_metadata(const_bytes(source, size),
                                   C.byref(limits) if limits is not None else None, C.byref(h))
    return Status(st), (ImageMetadata(h.value) if st == 0 else None)


class TiffCompression(enum.IntEnum):
    none = 0
    deflate = 1


def read_tiff(path, limits: TiffReadLimits | None = None):
    """io::read_tiff: (Status, image) where image is None or a dict with the ImageSpec fields,
    "pitch_bytes" and "pixels" (a (height, width) uint16 or float32 array)."""
    h = C.c_void_p(0)
    st = N.lib().ts_read_tiff(os.fsencode(path), C.byref(limits) if limits is not None else None,
                              C.byref(h))
    if st != 0:
        return Status(st), None
    try:
        spec, pitch, data, size = ImageSpec(), C.c_uint64(), C.c_void_p(), C.c_uint64()
        N.lib().ts_tiff_image_pixels(h.value, C.byref(spec), C.byref(pitch), C.byref(data),
                                     C.byref(size))
        raw = np.ctypeslib.as_array(C.cast(data, C.POINTER(C.c_uint8)), (size.value,)).copy()
    finally:
        N.lib().ts_tiff_image_destroy(h.value)
    dtype = np.uint16 if spec.type == PixelType.uint16 else np.float32
    pixels = raw.view(dtype).reshape(spec.height, spec.width)
    return Status(st), {"type": PixelType(spec.type), "width": spec.width,
                        "height": spec.height, "pitch_bytes": pitch.value, "pixels": pixels}


def write_tiff(path, image, options: TiffWriteOptions | None = None) -> Status:
    """io::write_tiff of a host image: a (height, width) uint16 or float32 array, or a
    ConstImageView of host memory."""
    if isinstance(image, np.ndarray):
        arr = np.ascontiguousarray(image)
        ptype = PixelType.uint16 if arr.dtype == np.uint16 else PixelType.float32
        v = const_view(arr, ptype, arr.shape[1], arr.shape[0])
        keep = arr  # noqa: F841  (alive across the call)
    else:
        v = image
    return Status(N.lib().ts_write_tiff(os.fsencode(path), v,
                                        C.byref(options) if options is not None else None))


def version() -> str:
    return N.lib().ts_version().decode()


def info_json() -> str:
    need = C.c_uint64(0)
    N.lib().ts_info_json(None, 0, C.byref(need))
    buf = C.create_string_buffer(need.value)
    N.lib().ts_info_json(buf, need.value, C.byref(need))
    return buf.value.decode()
