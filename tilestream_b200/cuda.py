"""Python mirror of include/tilestream/cuda.h: plan preparation and the five executors.

Device buffers are any objects with a device address (torch CUDA tensors, or addresses from
`allocate`); streams are CUDA stream handles (int) or torch.cuda.Stream objects.
"""
from __future__ import annotations

import ctypes as C
import enum

from . import _native as N
from .api import (BatchItem, BatchRequest, MutableBytes, ResultBuffer, Status, TileShape,
                  WorkspaceSpec, workspace_size)


class Operation(enum.IntEnum):
    compress = 0
    decompress = 1
    decode_roi = 2
    calibrate = 3
    decode_calibrate = 4


class ParameterKind(enum.IntEnum):
    scalar = 0
    map = 1


def stream_handle(stream) -> int:
    if stream is None:
        return 0
    if hasattr(stream, "cuda_stream"):
        return int(stream.cuda_stream)
    return int(stream)


class BatchPlan:
    """An owned tilestream::cuda::BatchPlan."""

    def __init__(self, handle: int):
        self.handle = handle

    def workspace_spec(self) -> WorkspaceSpec:
        spec = WorkspaceSpec()
        N.lib().ts_plan_workspace_spec(self.handle, C.byref(spec))
        return spec

    def workspace_bytes(self) -> int:
        st, n = workspace_size(self.workspace_spec())
        if st != Status.success:
            raise RuntimeError(f"workspace_size: {st!r}")
        return n

    def __del__(self, _lib=N.lib):
        # _lib is bound at definition: module globals may already be gone at interpreter exit.
        if getattr(self, "handle", None):
            _lib().ts_plan_destroy(self.handle)
            self.handle = None


def make_request(operation, items, tile: TileShape | None = None) -> BatchRequest:
    items = list(items)
    arr = (BatchItem * max(1, len(items)))(*items)
    req = BatchRequest(int(operation), C.cast(arr, C.POINTER(BatchItem)) if items else None,
                       len(items), tile if tile is not None else TileShape())
    req._keep = arr  # the item array must outlive prepare_batch
    return req


def prepare_batch(request: BatchRequest, plan: BatchPlan | None = None, stream=None):
    """Returns (Status, plan). On failure the previous plan (if any) is returned unchanged."""
    h = C.c_void_p(0)
    st = N.lib().ts_prepare_batch(C.byref(request), C.byref(h), stream_handle(stream))
    if st == 0:
        return Status.success, BatchPlan(h.value)
    return Status(st), plan


def inspect_decode(request: BatchRequest):
    """Host-only planning of a decode request (ts_inspect_decode): (Status, [TaskSpan...]).
    No device is touched, so the request may carry stand-in addresses."""
    count = C.c_uint64(0)
    st = N.lib().ts_inspect_decode(C.byref(request), None, 0, C.byref(count))
    spans = (N.TaskSpan * max(1, count.value))()
    st = N.lib().ts_inspect_decode(C.byref(request), spans, count.value, C.byref(count))
    return Status(st), list(spans[:count.value])


def _results(results) -> ResultBuffer:
    if isinstance(results, ResultBuffer):
        return results
    from .api import _ptr, nbytes
    return ResultBuffer(_ptr(results), nbytes(results) // 16)


def _workspace(workspace) -> MutableBytes:
    if isinstance(workspace, MutableBytes):
        return workspace
    if workspace is None:
        return MutableBytes(None, 0)
    from .api import mutable_bytes
    return mutable_bytes(workspace)


def _executor(name):
    def run(plan: BatchPlan, workspace, results, stream=None) -> Status:
        fn = getattr(N.lib(), name)
        return Status(fn(plan.handle if plan is not None else None, _workspace(workspace),
                         _results(results), stream_handle(stream)))
    run.__name__ = name[3:]
    return run


compress_async = _executor("ts_compress_async")
decompress_async = _executor("ts_decompress_async")
decode_roi_async = _executor("ts_decode_roi_async")
calibrate_async = _executor("ts_calibrate_async")
decode_calibrate_async = _executor("ts_decode_calibrate_async")


def synchronize(stream=None) -> Status:
    return Status(N.lib().ts_synchronize(stream_handle(stream)))


def allocate(nbytes: int, stream=None):
    """DeviceBuffer::allocate: returns (Status, device address)."""
    p = C.c_void_p(0)
    st = N.lib().ts_device_allocate(nbytes, stream_handle(stream), C.byref(p))
    return Status(st), (p.value or 0)


def release(address: int, stream=None) -> Status:
    return Status(N.lib().ts_device_release(address, stream_handle(stream)))


# ---- mixed batches (include/tilestream/batch.h) ----------------------------------------------

class MixedBatch:
    """An owned tilestream::cuda::MixedBatch: many decodes of mixed pixel types, geometries and
    operations in one persistent kernel, replayed as a CUDA graph."""

    def __init__(self, handle: int, keep=()):
        self.handle = handle
        self._keep = keep

    def run(self, stream=None) -> Status:
        return Status(N.lib().ts_run_mixed_batch(self.handle, stream_handle(stream)))

    def stats(self) -> dict:
        s = N.MixedStats()
        N.lib().ts_mixed_batch_stats(self.handle, C.byref(s))
        return {"tiles": s.tiles, "shape": s.shape, "grid": s.grid, "per_sm": s.per_sm,
                "graph": bool(s.graph), "tuned_us": round(s.tuned_us, 2)}

    def __del__(self, _lib=N.lib):
        # _lib is bound at definition: module globals may already be gone at interpreter exit.
        if getattr(self, "handle", None):
            _lib().ts_mixed_batch_destroy(self.handle)
            self.handle = None


# ---- unparsed files (include/tilestream/unparsed.h) -------------------------------------------

MAX_UNPARSED_FILES = 16


def decode_unparsed_async(files, results, stream=None) -> Status:
    """Whole-image decode of .tsc files never parsed on the host. files: a sequence of
    (device ConstBytes of the whole file, host copy of its first 64 bytes (bytes or uint8
    array), ImageView of the device output). results: ResultBuffer or a device buffer."""
    files = list(files)
    arr = (N.UnparsedFile * max(1, len(files)))()
    keep = []
    for k, (src, header, out) in enumerate(files):
        head = C.create_string_buffer(bytes(header[:64]) if len(header) >= 64 else bytes(header),
                                      64)
        keep.append(head)
        arr[k].bytes = src
        arr[k].header = C.cast(head, C.c_void_p)
        arr[k].output = out
    return Status(N.lib().ts_decode_unparsed_async(arr, len(files), _results(results),
                                                   stream_handle(stream)))


def decode_shape_count() -> int:
    return int(N.lib().ts_decode_shape_count())


def prepare_mixed_batch(items, results, stream=None, graph=True, autotune=False,
                        tune_cache=None, shape=-1):
    """items: iterable of (Operation, BatchItem). Returns (Status, MixedBatch or None).
    shape >= 0 fixes the kernel shape (no tuning)."""
    items = list(items)
    arr = (N.MixedItem * max(1, len(items)))(*[N.MixedItem(int(op), it) for op, it in items])
    opts = N.MixedOptions(1 if graph else 0, 1 if autotune else 0,
                          tune_cache.encode() if tune_cache else None, int(shape))
    h = C.c_void_p(0)
    st = N.lib().ts_prepare_mixed_batch(arr, len(items), _results(results), C.byref(opts),
                                        C.byref(h), stream_handle(stream))
    if st == 0:
        return Status.success, MixedBatch(h.value)
    return Status(st), None


class Server:
    """An owned tilestream::cuda::Server: archives resident in device memory, ROI and
    calibrated-ROI requests admitted by output-pool memory and batched into the persistent
    decoder, several batches in flight (continuous batching).

    Archives are added with their device bytes and parsed metadata (both kept alive here),
    then sealed; run() serves a request stream and returns (Status, outcomes, stats)."""

    def __init__(self, pool_bytes=1 << 30, max_batch=48, max_inflight=4, max_batch_tiles=1 << 22,
                 retain_outputs=False, serial=False):
        self.options = N.ServeOptions(pool_bytes, max_batch, max_inflight, max_batch_tiles,
                                      1 if retain_outputs else 0, 1 if serial else 0)
        h = C.c_void_p(0)
        st = N.lib().ts_server_create(C.byref(self.options), C.byref(h))
        if st != 0:
            raise RuntimeError(f"ts_server_create: {Status(st).name}")
        self.handle = h.value
        self._keep = []

    def add_archive(self, device_bytes, metadata, owner=None) -> tuple[Status, int]:
        """device_bytes: ConstBytes of the archive in device memory; metadata: a parsed
        ImageMetadata (api.parse_metadata); owner: the object holding the device memory (kept
        alive with the server)."""
        i = C.c_uint32(0)
        st = N.lib().ts_server_add_archive(self.handle, device_bytes, metadata.handle,
                                           C.byref(i))
        if st == 0:
            self._keep.append((owner, metadata))
        return Status(st), i.value

    def seal(self) -> Status:
        return Status(N.lib().ts_server_seal(self.handle))

    def pool(self) -> N.MutableBytes:
        p = N.MutableBytes()
        N.lib().ts_server_pool(self.handle, C.byref(p))
        return p

    def run(self, requests):
        """requests: a sequence of N.ServeRequest or a ctypes array of them."""
        if isinstance(requests, C.Array):
            arr, count = requests, len(requests)
        else:
            requests = list(requests)
            arr = (N.ServeRequest * max(1, len(requests)))(*requests)
            count = len(requests)
        outcomes = (N.ServeOutcome * max(1, count))()
        stats = N.ServeStats()
        st = N.lib().ts_server_run(self.handle, arr, count, outcomes, C.byref(stats))
        return Status(st), outcomes, stats

    # Sessions: requests submitted while the serving loop runs on a thread of its own. The
    # native calls release the GIL, so producers and consumers may be Python threads.
    def start(self, max_outstanding=4096) -> Status:
        return Status(N.lib().ts_server_start(self.handle, max_outstanding))

    def submit(self, request) -> tuple[Status, int]:
        """request: an N.ServeRequest (arrival_us ignored). Returns (Status, ticket)."""
        t = C.c_uint64(0)
        st = N.lib().ts_server_submit(self.handle, C.byref(request), C.byref(t))
        return Status(st), t.value

    def wait(self, ticket, timeout_us=1_000_000):
        """(Status, done, ServeOutcome): done is False when timeout_us passed first."""
        out = N.ServeOutcome()
        done = C.c_int(0)
        st = N.lib().ts_server_wait(self.handle, ticket, timeout_us, C.byref(out), C.byref(done))
        return Status(st), bool(done.value), out

    def release(self, ticket) -> Status:
        return Status(N.lib().ts_server_release(self.handle, ticket))

    def stop(self) -> Status:
        return Status(N.lib().ts_server_stop(self.handle))

    def __del__(self, _lib=N.lib):
        # _lib is bound at definition: module globals may already be gone at interpreter exit.
        if getattr(self, "handle", None):
            _lib().ts_server_destroy(self.handle)
            self.handle = None


# ---- ROI staging from an archive outside the GPU (include/tilestream/staging.h) ---------------

def roi_staging_size(metadata, roi):
    """(Status, RoiStaging): the tiles, payload bytes and copies of staging `roi`."""
    out = N.RoiStaging()
    st = N.lib().ts_roi_staging_size(metadata.handle, roi, C.byref(out))
    return Status(st), out


def stage_roi_tiles(metadata, roi, archive, staging, mappings, stream=None):
    """Enqueues the copies of the ROI's tile payloads from `archive` (ConstBytes of the whole
    file, pinned host or device memory) into `staging` (MutableBytes of device memory) and fills
    `mappings` (a ctypes array of TileMapping). Returns (Status, RoiStaging)."""
    out = N.RoiStaging()
    st = N.lib().ts_stage_roi_tiles(metadata.handle, roi, archive, staging, mappings,
                                    len(mappings), stream_handle(stream), C.byref(out))
    return Status(st), out


def serve_requests(stream: dict, scale_arrivals: float = 1.0):
    """A ctypes array of ServeRequest from the arrays of workloads.serving_requests."""
    n = len(stream["arrival_us"])
    arr = (N.ServeRequest * max(1, n))()
    for i in range(n):
        r = arr[i]
        r.archive = int(stream["archive"][i])
        r.roi = N.Roi(int(stream["x"][i]), int(stream["y"][i]), int(stream["width"][i]),
                      int(stream["height"][i]))
        r.calibrated = 1 if stream["calibrated"][i] else 0
        r.offset = float(stream["offset"][i])
        r.gain = float(stream["gain"][i])
        r.arrival_us = float(stream["arrival_us"][i]) * scale_arrivals
    return arr if n else (N.ServeRequest * 0)()
