"""ctypes declarations of include/tilestream_c.h and the loader of libtilestream_b200.so.

The library is built in-tree (tilestream_b200/build.py). Loading never falls back to anything
else: if the library cannot be built or loaded, importing the API raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

from . import build as _build

u8, u16, u32, u64 = C.c_uint8, C.c_uint16, C.c_uint32, C.c_uint64
vp = C.c_void_p


class ImageSpec(C.Structure):
    _fields_ = [("type", u32), ("width", u32), ("height", u32)]


class TileShape(C.Structure):
    _fields_ = [("width", u16), ("height", u16)]

    def __init__(self, width=128, height=32):
        super().__init__(width, height)


class Roi(C.Structure):
    _fields_ = [("x", u32), ("y", u32), ("width", u32), ("height", u32)]


class ConstBytes(C.Structure):
    _fields_ = [("data", vp), ("size", u64)]


class MutableBytes(C.Structure):
    _fields_ = [("data", vp), ("size", u64)]


class ConstImageView(C.Structure):
    _fields_ = [("data", vp), ("image", ImageSpec), ("pitch_bytes", u64),
                ("capacity_bytes", u64)]


class ImageView(C.Structure):
    _fields_ = [("data", vp), ("image", ImageSpec), ("pitch_bytes", u64),
                ("capacity_bytes", u64)]


class DeviceResult(C.Structure):
    _fields_ = [("status", u32), ("reserved", u32), ("bytes_written", u64)]


class Parameter(C.Structure):
    _fields_ = [("kind", u32), ("scalar", C.c_float), ("map", ConstImageView)]


class Calibration(C.Structure):
    _fields_ = [("offset", Parameter), ("gain", Parameter)]

    def __init__(self, *args, **kw):
        super().__init__(*args, **kw)
        if not args and "gain" not in kw:
            self.gain.scalar = 1.0


class TileMapping(C.Structure):
    _fields_ = [("tile_index", u64), ("input_offset", u64)]


class ParseLimits(C.Structure):
    _fields_ = [("file_bytes", u64), ("tile_count", u64), ("metadata_bytes", u64)]


class UnparsedFile(C.Structure):
    _fields_ = [("bytes", ConstBytes), ("header", C.c_void_p), ("output", ImageView)]


class TiffReadLimits(C.Structure):
    _fields_ = [("max_width", u32), ("max_height", u32), ("max_decoded_bytes", u64)]

    def __init__(self, *args, **kw):
        super().__init__(*args, **kw)
        if not args and not kw:
            self.max_width = self.max_height = 0xFFFFFFFF
            self.max_decoded_bytes = (1 << 63) - 1


class TiffWriteOptions(C.Structure):
    _fields_ = [("bigtiff", u32), ("compression", u32), ("horizontal_predictor", u32),
                ("tile_width", u32), ("tile_height", u32), ("deflate_level", u32)]

    def __init__(self, *args, **kw):
        super().__init__(*args, **kw)
        if not args:
            for k, v in (("tile_width", 128), ("tile_height", 32), ("deflate_level", 6)):
                if k not in kw:
                    setattr(self, k, v)


class WorkspaceSpec(C.Structure):
    _fields_ = [("image_count", u64), ("tile_count", u64), ("tile", TileShape),
                ("scan_temp_bytes", u64)]


class TileMetadata(C.Structure):
    _fields_ = [("mode", u32), ("width", u16), ("height", u16), ("offset", u64),
                ("length", u64), ("first_segment", u64)]


class SegmentMetadata(C.Structure):
    _fields_ = [("seed", u32), ("bit_width", u32), ("payload_offset", u64),
                ("payload_bytes", u64)]


class CompressedInput(C.Structure):
    _fields_ = [("bytes", ConstBytes), ("metadata", vp), ("mappings", C.POINTER(TileMapping)),
                ("mapping_count", u64), ("encoder_result", vp), ("trusted_image", ImageSpec),
                ("trusted_tile", TileShape)]


class BatchItem(C.Structure):
    _fields_ = [("input", ConstImageView), ("output", ImageView),
                ("compressed_output", MutableBytes), ("compressed_input", CompressedInput),
                ("roi", Roi), ("calibration", Calibration)]


class BatchRequest(C.Structure):
    _fields_ = [("operation", u32), ("items", C.POINTER(BatchItem)), ("count", u64),
                ("tile", TileShape)]


class ResultBuffer(C.Structure):
    _fields_ = [("data", vp), ("count", u64)]


class TaskSpan(C.Structure):
    _fields_ = [("image", u64), ("read_begin", u64), ("read_end", u64), ("write_begin", u64),
                ("write_end", u64), ("rows_end", u64), ("mode", u32), ("flags", u32),
                ("width", u32), ("height", u32)]


class MixedItem(C.Structure):
    _fields_ = [("operation", u32), ("item", BatchItem)]


class MixedOptions(C.Structure):
    _fields_ = [("graph", u32), ("autotune", u32), ("tune_cache", C.c_char_p),
                ("shape", C.c_int32)]


class MixedStats(C.Structure):
    _fields_ = [("tiles", u64), ("shape", u32), ("grid", u32), ("per_sm", u32), ("graph", u32),
                ("tuned_us", C.c_float)]


class RoiStaging(C.Structure):
    _fields_ = [("tiles", u64), ("bytes", u64), ("copies", u64)]


class ServeRequest(C.Structure):
    _fields_ = [("archive", u32), ("roi", Roi), ("calibrated", u32), ("offset", C.c_float),
                ("gain", C.c_float), ("arrival_us", C.c_double)]


class ServeOptions(C.Structure):
    _fields_ = [("output_pool_bytes", u64), ("max_batch", u32), ("max_inflight", u32),
                ("max_batch_tiles", u64), ("retain_outputs", u32), ("serial", u32)]


class ServeStats(C.Structure):
    _fields_ = [(name, C.c_double) for name in
                ("wall_us", "throughput_rps", "decoded_gbs", "p50_us", "p90_us", "p99_us",
                 "max_us", "mean_us")] + \
               [("completed", u64), ("rejected", u64), ("batches", u64),
                ("mean_batch", C.c_double), ("max_inflight", u64), ("stalls", u64),
                ("tiles", u64), ("output_bytes", u64)]


class ServeOutcome(C.Structure):
    _fields_ = [("latency_us", C.c_double), ("queued_us", C.c_double), ("output_offset", u64),
                ("output_pitch", u64), ("batch_size", u32), ("result", DeviceResult)]


_SIGNATURES = {
    "ts_image_span": (C.c_int, [ImageSpec, u64, C.POINTER(u64)]),
    "ts_compress_bound": (C.c_int, [ImageSpec, TileShape, C.POINTER(u64)]),
    "ts_workspace_size": (C.c_int, [C.POINTER(WorkspaceSpec), C.POINTER(u64)]),
    "ts_parse_metadata": (C.c_int, [ConstBytes, C.POINTER(ParseLimits), C.POINTER(vp)]),
    "ts_metadata_create": (C.c_int, [ImageSpec, TileShape, u64, vp, u64, vp, u64,
                                     C.POINTER(vp)]),
    "ts_metadata_destroy": (None, [vp]),
    "ts_metadata_info": (None, [vp, C.POINTER(ImageSpec), C.POINTER(TileShape), C.POINTER(u64),
                                C.POINTER(u64), C.POINTER(u64)]),
    "ts_metadata_tiles": (vp, [vp]),
    "ts_metadata_segments": (vp, [vp]),
    "ts_cpu_compress": (C.c_int, [ConstImageView, TileShape, MutableBytes, C.POINTER(u64)]),
    "ts_cpu_decompress": (C.c_int, [ConstBytes, ImageView, C.POINTER(ParseLimits)]),
    "ts_prepare_batch": (C.c_int, [C.POINTER(BatchRequest), C.POINTER(vp), vp]),
    "ts_plan_destroy": (None, [vp]),
    "ts_inspect_decode": (C.c_int, [C.POINTER(BatchRequest), C.POINTER(TaskSpan), u64,
                                    C.POINTER(u64)]),
    "ts_plan_workspace_spec": (C.c_int, [vp, C.POINTER(WorkspaceSpec)]),
    "ts_compress_async": (C.c_int, [vp, MutableBytes, ResultBuffer, vp]),
    "ts_decompress_async": (C.c_int, [vp, MutableBytes, ResultBuffer, vp]),
    "ts_decode_roi_async": (C.c_int, [vp, MutableBytes, ResultBuffer, vp]),
    "ts_calibrate_async": (C.c_int, [vp, MutableBytes, ResultBuffer, vp]),
    "ts_decode_calibrate_async": (C.c_int, [vp, MutableBytes, ResultBuffer, vp]),
    "ts_prepare_mixed_batch": (C.c_int, [C.POINTER(MixedItem), u64, ResultBuffer,
                                         C.POINTER(MixedOptions), C.POINTER(vp), vp]),
    "ts_run_mixed_batch": (C.c_int, [vp, vp]),
    "ts_decode_shape_count": (u32, []),
    "ts_mixed_batch_stats": (C.c_int, [vp, C.POINTER(MixedStats)]),
    "ts_mixed_batch_destroy": (None, [vp]),
    "ts_server_create": (C.c_int, [C.POINTER(ServeOptions), C.POINTER(vp)]),
    "ts_server_add_archive": (C.c_int, [vp, ConstBytes, vp, C.POINTER(u32)]),
    "ts_server_seal": (C.c_int, [vp]),
    "ts_server_run": (C.c_int, [vp, C.POINTER(ServeRequest), u64, C.POINTER(ServeOutcome),
                                C.POINTER(ServeStats)]),
    "ts_server_pool": (C.c_int, [vp, C.POINTER(MutableBytes)]),
    "ts_server_start": (C.c_int, [vp, u32]),
    "ts_server_submit": (C.c_int, [vp, C.POINTER(ServeRequest), C.POINTER(u64)]),
    "ts_server_wait": (C.c_int, [vp, u64, u64, C.POINTER(ServeOutcome), C.POINTER(C.c_int)]),
    "ts_server_release": (C.c_int, [vp, u64]),
    "ts_server_stop": (C.c_int, [vp]),
    "ts_server_destroy": (None, [vp]),
    "ts_roi_staging_size": (C.c_int, [vp, Roi, C.POINTER(RoiStaging)]),
    "ts_stage_roi_tiles": (C.c_int, [vp, Roi, ConstBytes, MutableBytes, C.POINTER(TileMapping),
                                     u64, vp, C.POINTER(RoiStaging)]),
    "ts_decode_unparsed_async": (C.c_int, [C.POINTER(UnparsedFile), u64, ResultBuffer, vp]),
    "ts_read_tiff": (C.c_int, [C.c_char_p, C.POINTER(TiffReadLimits), C.POINTER(vp)]),
    "ts_tiff_image_pixels": (C.c_int, [vp, C.POINTER(ImageSpec), C.POINTER(u64),
                                       C.POINTER(vp), C.POINTER(u64)]),
    "ts_tiff_image_destroy": (None, [vp]),
    "ts_write_tiff": (C.c_int, [C.c_char_p, ConstImageView, C.POINTER(TiffWriteOptions)]),
    "ts_compress_noalloc": (C.c_int, [ConstImageView, TileShape, MutableBytes, vp, vp]),
    "ts_compress_noalloc_max_tiles": (u64, []),
    "ts_device_allocate": (C.c_int, [u64, vp, C.POINTER(vp)]),
    "ts_device_release": (C.c_int, [vp, vp]),
    "ts_synchronize": (C.c_int, [vp]),
    "ts_version": (C.c_char_p, []),
    "ts_info_json": (C.c_int, [C.c_char_p, u64, C.POINTER(u64)]),
}

_lib = None
_lock = threading.Lock()


def library_path() -> str:
    return _build.LIB


def lib() -> C.CDLL:
    """The loaded library (built first when its sources changed)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            path = _build.build()
            if not os.path.exists(path):
                raise ImportError(f"libtilestream_b200.so missing at {path}")
            handle = C.CDLL(path)
            for name, (restype, argtypes) in _SIGNATURES.items():
                fn = getattr(handle, name)
                fn.restype = restype
                fn.argtypes = argtypes
            _lib = handle
    return _lib
