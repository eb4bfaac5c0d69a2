"""Shared helpers of the tests: device round trips through the library's C ABI, with torch
providing device memory and streams only."""
from __future__ import annotations

import numpy as np

from tilestream_b200 import api, cuda
from tilestream_b200.api import (BatchItem, Calibration, CompressedInput, ConstBytes, Roi,
                                 Status, TileMapping, TileShape)

SENTINEL = 0xA5


def torch():
    import torch as t
    return t


def to_device(array: np.ndarray):
    t = torch()
    flat = np.ascontiguousarray(array).view(np.uint8).reshape(-1)
    return t.from_numpy(flat.copy()).to("cuda")


def device_bytes(n: int, fill: int | None = SENTINEL):
    t = torch()
    buf = t.empty(max(n, 1), dtype=t.uint8, device="cuda")
    if fill is not None:
        buf.fill_(fill)
    return buf


def host(buf) -> np.ndarray:
    return buf.cpu().numpy()


class Run:
    """One prepared plan with its workspace and results, executed on torch's current stream."""

    def __init__(self, operation, items, tile=None, keep=()):
        t = torch()
        self.keep = list(keep)
        self.count = len(items)
        self.stream = t.cuda.current_stream()
        self.request = cuda.make_request(operation, items, tile)
        self.status, self.plan = cuda.prepare_batch(self.request, None, self.stream)
        self.workspace = None
        self.results = None
        if self.status == Status.success:
            nbytes = self.plan.workspace_bytes()
            self.workspace = t.empty(max(nbytes, 256), dtype=t.uint8, device="cuda")
            self.results = device_bytes(16 * max(self.count, 1), fill=0xFF)

    def execute(self, executor) -> Status:
        ws = api.MutableBytes(self.workspace.data_ptr(), self.workspace.numel())
        return executor(self.plan, ws, self.results, self.stream)

    def records(self):
        torch().cuda.synchronize()
        raw = host(self.results).view(np.uint32).reshape(-1, 4)[:self.count]
        return [(int(r[0]), int(r[1]), int(r[2]) | (int(r[3]) << 32)) for r in raw]


def parsed_source(file: bytes):
    st, meta = api.parse_metadata(file)
    assert st == Status.success, st
    dev = to_device(np.frombuffer(file, dtype=np.uint8))
    src = CompressedInput()
    src.bytes = ConstBytes(dev.data_ptr(), len(file))
    src.metadata = meta.handle
    return src, meta, dev


def decode_item(src, ptype, out_dev, width, height, pitch, roi=None, calibration=None):
    item = BatchItem()
    item.compressed_input = src
    item.output = api.view(out_dev, ptype, width, height, pitch, out_dev.numel())
    if roi is not None:
        item.roi = Roi(*roi)
    if calibration is not None:
        item.calibration = calibration
    return item


def gpu_decode(file: bytes, roi=None, pitch=None, operation=None, calibration=None,
               out_type=None):
    """Decodes one parsed archive on the GPU. Returns (status, record, output bytes, pitch)."""
    src, meta, dev = parsed_source(file)
    image = meta.image
    ptype = api.PixelType(image.type)
    if roi is None:
        roi = (0, 0, image.width, image.height)
        op = cuda.Operation.decompress if operation is None else operation
    else:
        op = cuda.Operation.decode_roi if operation is None else operation
    otype = out_type or (api.PixelType.float32 if op == cuda.Operation.decode_calibrate else ptype)
    w, h = roi[2], roi[3]
    pitch = pitch if pitch is not None else w * api.sample_bytes(otype)
    out = device_bytes(pitch * h)
    item = decode_item(src, otype, out, w, h, pitch, roi if op != cuda.Operation.decompress
                       else None, calibration)
    run = Run(op, [item], keep=[meta, dev, out])
    if run.status != Status.success:
        return run.status, None, None, pitch
    executor = {cuda.Operation.decompress: cuda.decompress_async,
                cuda.Operation.decode_roi: cuda.decode_roi_async,
                cuda.Operation.decode_calibrate: cuda.decode_calibrate_async}[op]
    st = run.execute(executor)
    assert st == Status.success, st
    rec = run.records()[0]
    return st, rec, host(out), pitch


def logical(buf: np.ndarray, width: int, height: int, pitch: int, s: int) -> np.ndarray:
    """The logical pixel bytes of a pitched buffer, rows concatenated."""
    rows = [buf[y * pitch: y * pitch + width * s] for y in range(height)]
    return np.concatenate(rows) if rows else np.zeros(0, np.uint8)


def padding_untouched(buf: np.ndarray, width: int, height: int, pitch: int, s: int) -> bool:
    for y in range(height):
        pad = buf[y * pitch + width * s: (y + 1) * pitch]
        if pad.size and not np.all(pad == SENTINEL):
            return False
    tail = buf[height * pitch:]
    return bool(np.all(tail == SENTINEL)) if tail.size else True


def crop(pixels: np.ndarray, pitch: int, s: int, roi) -> np.ndarray:
    x, y, w, h = roi
    rows = [pixels[(y + r) * pitch + x * s:(y + r) * pitch + (x + w) * s] for r in range(h)]
    return np.concatenate(rows)


def read_device(address: int, nbytes: int) -> np.ndarray:
    """nbytes of device memory at a raw address (memory the library owns, such as a server's
    output pool), copied to the host through the CUDA runtime that torch has loaded."""
    import ctypes
    t = torch()
    t.cuda.synchronize()
    rt = ctypes.CDLL("libcudart.so.12")
    out = np.empty(max(nbytes, 1), np.uint8)
    rc = rt.cudaMemcpy(ctypes.c_void_p(out.ctypes.data), ctypes.c_void_p(address),
                       ctypes.c_size_t(nbytes), 2)  # cudaMemcpyDeviceToHost
    assert rc == 0, rc
    return out[:nbytes]
