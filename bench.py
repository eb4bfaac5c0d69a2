"""Benchmark of the TileStream GPU codec path on B200.

Workload (the config the headline metric is quoted on, fits one GPU): a uint16 4096x4096 detector
frame (seeded synthetic generator, seed 2) encoded with tiles 128x32, 64x64 and 256x16. One step
decodes the three archives device-to-device (one decompress_async each). Inputs and outputs rotate
over R copies so that every step reads archives that are not L2-resident (the rotation set is
larger than the 126 MB L2). The step is captured once as a CUDA graph and replayed.

Reported: decoded-pixel GB/s (value), the decoder's HBM roofline fraction, an end-to-end figure
through the C ABI with pinned host buffers (H2D of the archive, decode, D2H of the pixels, every
step), the reference CPU codec on the host cores, and SM clocks sampled during the timed region.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: archives are independent, so N ranks each decode their own copies (weak scaling, no
collective); the timed region is bracketed by a barrier and the max over ranks is reported.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GPU decode GB/s (decoded uint16 pixels, 4096x4096 frame x 3 tile shapes)"
SHAPES = ((128, 32), (64, 64), (256, 16))
W = H = 4096
SEED = 2


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, burst copy)"
    return 6650.0, "fallback (6.65 TB/s, earlier measurement on this pool)"


def ncu_traffic():
    """DRAM bytes per decode launch from the committed ncu summary, when present."""
    path = os.path.join(ROOT, "profiles", "decode_c2_u16_4096.md")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        for line in f:
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1].strip())
    return None


class ClockSampler:
    """Samples SM clock and throttle reasons with NVML while the timed region runs."""

    def __init__(self, index: int, period: float = 0.005):
        self.index, self.period = index, period
        self.samples, self.reasons = [], set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._thread = None

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            self.handle = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM)
        except Exception:  # noqa: BLE001 - clocks are reported as unavailable
            self.nvml = None
            return self
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()
        return self

    def _run(self):
        nv = self.nvml
        names = {
            "hw_slowdown": getattr(nv, "nvmlClocksEventReasonHwSlowdown", 0x8),
            "sw_thermal_slowdown": getattr(nv, "nvmlClocksEventReasonSwThermalSlowdown", 0x20),
            "hw_thermal_slowdown": getattr(nv, "nvmlClocksEventReasonHwThermalSlowdown", 0x40),
            "sw_power_cap": getattr(nv, "nvmlClocksEventReasonSwPowerCap", 0x4),
        }
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.handle, nv.NVML_CLOCK_SM))
                mask = nv.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
                for name, bit in names.items():
                    if mask & bit:
                        self.reasons.add(name)
            except Exception:  # noqa: BLE001
                pass
            time.sleep(self.period)

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread:
            self._thread.join()
        return False

    def report(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unavailable"]}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "samples": len(self.samples), "reasons": sorted(self.reasons)}


def cpu_decode_rate(archive: bytes, seconds: float, threads: int, use_reference: bool):
    """Decoded bytes/s of the CPU codec on `threads` host threads, one image per thread."""
    import oracle
    codec = oracle.Reference() if use_reference else oracle.Oracle()
    stop = time.perf_counter() + seconds
    done = [0] * threads

    def worker(k):
        out = np.empty(W * H * 2, dtype=np.uint8)
        while time.perf_counter() < stop:
            if use_reference:
                st, _ = codec.decompress(archive, 1, W, H, out=out)
            else:
                st, _ = codec.decompress(archive, 1, W, H)
            assert st == 0
            done[k] += 1

    pool = [threading.Thread(target=worker, args=(k,)) for k in range(threads)]
    t0 = time.perf_counter()
    for t in pool:
        t.start()
    for t in pool:
        t.join()
    elapsed = time.perf_counter() - t0
    return sum(done) * W * H * 2 / elapsed, sum(done)


def prepare_workload(torch, stream, copies: int):
    """GPU-encoded archives (checked byte-identical to the CPU codec in the tests) and plans."""
    from tilestream_b200 import api, cuda, workloads
    from tilestream_b200.api import BatchItem, CompressedInput, ConstBytes, Status, TileShape

    frame = workloads.detector_frame(W, H, seed=SEED)
    dev_frame = torch.from_numpy(frame.view(np.uint8).reshape(-1).copy()).cuda()
    shapes = []
    for tile in SHAPES:
        st, bound = api.compress_bound(api.image_spec(1, W, H), TileShape(*tile))
        archive = torch.empty(bound, dtype=torch.uint8, device="cuda")
        item = BatchItem()
        item.input = api.const_view(dev_frame, 1, W, H, W * 2)
        item.compressed_output = api.MutableBytes(archive.data_ptr(), bound)
        st, plan = cuda.prepare_batch(cuda.make_request(cuda.Operation.compress, [item],
                                                        TileShape(*tile)), None, stream)
        assert st == Status.success, st
        ws = torch.empty(plan.workspace_bytes(), dtype=torch.uint8, device="cuda")
        res = torch.zeros(16, dtype=torch.uint8, device="cuda")
        assert cuda.compress_async(plan, ws, res, stream) == Status.success
        torch.cuda.synchronize()
        size = int(res.cpu().numpy().view(np.uint64)[1])
        file = archive[:size].cpu().numpy().tobytes()
        st, meta = api.parse_metadata(file)
        assert st == Status.success
        tiles = meta.tiles
        algorithmic = int(tiles["length"].sum()) + 32 * len(tiles) + W * H * 2
        shapes.append({"tile": tile, "file": file, "meta": meta, "algorithmic": algorithmic})
        del ws, archive

    decode_ws = 0
    for s in shapes:
        s["copies"] = []
        for _ in range(copies):
            src_dev = torch.from_numpy(np.frombuffer(s["file"], dtype=np.uint8).copy()).cuda()
            out = torch.empty(W * H * 2, dtype=torch.uint8, device="cuda")
            src = CompressedInput()
            src.bytes = ConstBytes(src_dev.data_ptr(), len(s["file"]))
            src.metadata = s["meta"].handle
            item = BatchItem()
            item.compressed_input = src
            item.output = api.view(out, 1, W, H, W * 2)
            st, plan = cuda.prepare_batch(cuda.make_request(cuda.Operation.decompress, [item]),
                                          None, stream)
            assert st == Status.success, st
            decode_ws = max(decode_ws, plan.workspace_bytes())
            s["copies"].append({"src": src_dev, "out": out, "plan": plan})
    workspace = torch.empty(max(decode_ws, 256), dtype=torch.uint8, device="cuda")
    results = torch.zeros(16 * 3, dtype=torch.uint8, device="cuda")
    return frame, shapes, workspace, results


def run_ours(args, rank, world, device, torch, dist):
    from tilestream_b200 import api, cuda
    from tilestream_b200.api import Status

    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    copies = args.copies
    frame, shapes, workspace, results = prepare_workload(torch, stream, copies)
    wsb = api.MutableBytes(workspace.data_ptr(), workspace.numel())
    recs = [api.ResultBuffer(results.data_ptr() + 16 * k, 1) for k in range(3)]

    def enqueue(step):
        for k, s in enumerate(shapes):
            c = s["copies"][step % copies]
            st = cuda.decompress_async(c["plan"], wsb, recs[k], stream)
            assert st == Status.success, st

    # One graph per rotation slot: the three decodes of that slot. The executors validate
    # pointers with cudaPointerGetAttributes on the host, which global-mode capture rejects, so
    # capture is relaxed (the validation runs once, at capture time).
    graphs, capture_error = [], None
    try:
        for slot in range(copies):
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=stream, capture_error_mode="relaxed"):
                enqueue(slot)
            graphs.append(g)
    except Exception as e:  # noqa: BLE001 - recorded in the JSON line, launches stay eager
        capture_error = str(e).splitlines()[0]
        print(f"graph capture failed, timing eager launches: {capture_error}", file=sys.stderr)
        graphs = None
    torch.cuda.synchronize()

    def replay(i):
        if graphs is not None:
            graphs[i % copies].replay()
        else:
            enqueue(i % copies)

    # Correctness of the benchmarked outputs (one slot per shape).
    enqueue(0)
    torch.cuda.synchronize()
    for s in shapes:
        assert np.array_equal(s["copies"][0]["out"].cpu().numpy().view(np.uint16),
                              frame.reshape(-1)), "decode mismatch"
    r = results.cpu().numpy().view(np.uint64).reshape(3, 2)
    assert all(int(r[k, 0]) == 0 and int(r[k, 1]) == W * H * 2 for k in range(3)), r

    for i in range(args.warmup):
        replay(i)
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(device) as clocks:
        start.record(stream)
        for i in range(args.steps):
            replay(i)
        end.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = start.elapsed_time(end)
    if world > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    step_ms = ms / args.steps
    decoded_per_step = 3 * W * H * 2
    value = decoded_per_step * args.steps * world / (ms / 1e3) / 1e9

    # Per-shape device time (outside the timed region, same method).
    per_shape = {}
    for k, s in enumerate(shapes):
        def shape_pass(k=k, s=s):
            for slot in range(copies):
                cuda.decompress_async(s["copies"][slot]["plan"], wsb, recs[k], stream)
        g = None
        if graphs is not None:
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=stream, capture_error_mode="relaxed"):
                shape_pass()
        run_pass = g.replay if g is not None else shape_pass
        for _ in range(3):
            run_pass()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 20
        e0.record(stream)
        for _ in range(reps):
            run_pass()
        e1.record(stream)
        torch.cuda.synchronize()
        launch_ms = e0.elapsed_time(e1) / (reps * copies)
        per_shape["%dx%d" % s["tile"]] = {
            "launch_us": round(launch_ms * 1e3, 2),
            "decoded_gbs": round(W * H * 2 / launch_ms / 1e6, 1),
            "hbm_gbs": round(s["algorithmic"] / launch_ms / 1e6, 1),
            "file_bytes": len(s["file"]),
        }

    peak, peak_src = measured_peaks()
    alg_per_launch = statistics.mean(s["algorithmic"] for s in shapes)
    launch_ms = step_ms / 3
    achieved = alg_per_launch / (launch_ms / 1e3) / 1e9

    # End to end through the C ABI: pinned host archive -> device -> decode -> pinned host pixels.
    e2e = run_e2e(args, torch, stream, shapes, wsb, recs)

    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(step_ms, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16",
        "data": "synthetic (seeded detector frame generator, seed 2)",
        "config": {"workload": "uint16 4096x4096 frame, tiles 128x32 + 64x64 + 256x16, "
                               "device-to-device whole-image decode",
                   "images_per_step": 3, "rotation_copies": copies,
                   "l2": f"inputs rotate over {copies} copies "
                         f"({copies * sum(len(s['file']) + W * H * 2 for s in shapes) / 1e6:.0f} MB"
                         " > 126 MB L2)",
                   "parallelism": f"replicas{world}" if world > 1 else "single"},
        "gpu_launches": 3 * args.steps,
        "cuda_graph": graphs is not None,
        **({"graph_capture_error": capture_error} if capture_error else {}),
        "per_shape": per_shape,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                     "peak_source": peak_src, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "algorithmic_bytes_per_launch": int(alg_per_launch),
                     "traffic": ncu_traffic(), "kernel": "decode_kernel"},
        "e2e": e2e,
        "clocks": clocks.report(),
    }
    return line, shapes


def run_e2e(args, torch, stream, shapes, wsb, recs):
    """Per step: H2D copy of the three archives from pinned memory, three decodes, D2H copy of
    the three decoded frames into pinned memory."""
    from tilestream_b200 import cuda
    pinned_in = [torch.from_numpy(np.frombuffer(s["file"], dtype=np.uint8).copy()).pin_memory()
                 for s in shapes]
    pinned_out = [torch.empty(W * H * 2, dtype=torch.uint8).pin_memory() for _ in shapes]
    slots = [s["copies"][0] for s in shapes]
    steps = max(3, min(args.steps, 50))

    def step():
        for k, (s, c) in enumerate(zip(shapes, slots)):
            c["src"][:len(s["file"])].copy_(pinned_in[k], non_blocking=True)
            cuda.decompress_async(c["plan"], wsb, recs[k], stream)
            pinned_out[k].copy_(c["out"], non_blocking=True)

    for _ in range(3):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    h2d = sum(len(s["file"]) for s in shapes)
    d2h = 3 * W * H * 2
    return {"value": round(3 * W * H * 2 * steps / (ms / 1e3) / 1e9, 2), "unit": "GB/s",
            "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": steps,
            "ms_per_step": round(ms / steps, 4)}


def cpu_baseline(shapes, seconds):
    import oracle
    archive = shapes[0]["file"]
    ref = oracle.Reference.available()
    threads = os.cpu_count() or 1
    rate, images = cpu_decode_rate(archive, seconds, threads, ref)
    return {"value": round(rate / 1e9, 3), "unit": "GB/s", "cores": threads,
            "kind": "reference" if ref else "port",
            "sample": f"{images} decodes of the 4096x4096 uint16 128x32 archive, one image per "
                      f"thread, {seconds:.0f} s"}


def run_reference(args):
    """The reference CPU codec (compiled from its sources into oracle/_ref, else the C oracle
    port) decoding the same archives on all host threads."""
    import oracle
    from tilestream_b200 import workloads
    frame = workloads.detector_frame(W, H, seed=SEED)
    ref = oracle.Reference.available()
    codec = oracle.Reference() if ref else oracle.Oracle()
    files = [codec.compress_image(frame, tile) for tile in SHAPES]
    threads = os.cpu_count() or 1
    per_step = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        done = [0] * threads

        def worker(k):
            # Every thread decodes one whole frame per step, cycling over the three archives.
            out = np.empty(W * H * 2, dtype=np.uint8)
            f = files[k % 3]
            if ref:
                st, _ = codec.decompress(f, 1, W, H, out=out)
            else:
                st, _ = codec.decompress(f, 1, W, H)
            assert st == 0
            done[k] += 1

        pool = [threading.Thread(target=worker, args=(k,)) for k in range(threads)]
        for t in pool:
            t.start()
        for t in pool:
            t.join()
        elapsed = time.perf_counter() - t0
        if i >= args.warmup:
            per_step.append((sum(done), elapsed))
    images = sum(d for d, _ in per_step)
    seconds = sum(e for _, e in per_step)
    value = images * W * H * 2 / seconds / 1e9
    return {
        "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(seconds / len(per_step) * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u16", "impl": "reference",
        "data": "synthetic (seeded detector frame generator, seed 2)",
        "config": {"workload": "uint16 4096x4096 frame, tiles 128x32 + 64x64 + 256x16, "
                               "whole-image decode", "images_per_step": threads},
        "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": threads,
                         "kind": "reference" if ref else "port",
                         "sample": f"{images} whole-frame decodes over {len(per_step)} steps"},
        "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def run_profile_case(kind: str, launches: int = 3):
    """A small case for ncu captures: one launch of `kind` over four 4096x4096 frames (about
    216 MB of decode traffic, more than the 126 MB L2), repeated `launches` times."""
    import torch
    from tilestream_b200 import api, cuda, workloads
    from tilestream_b200.api import BatchItem, CompressedInput, ConstBytes, Status, TileShape
    stream = torch.cuda.current_stream()
    frame = workloads.detector_frame(W, H, seed=SEED)
    if kind == "encode":
        items, keep = [], []
        for _ in range(4):
            src = torch.from_numpy(frame.view(np.uint8).reshape(-1).copy()).cuda()
            st, bound = api.compress_bound(api.image_spec(1, W, H), TileShape())
            out = torch.empty(bound, dtype=torch.uint8, device="cuda")
            item = BatchItem()
            item.input = api.const_view(src, 1, W, H, W * 2)
            item.compressed_output = api.MutableBytes(out.data_ptr(), bound)
            items.append(item)
            keep += [src, out]
        st, plan = cuda.prepare_batch(cuda.make_request(cuda.Operation.compress, items), None,
                                      stream)
        executor = cuda.compress_async
    else:
        import oracle
        file = oracle.Oracle().compress_image(frame, (128, 32))
        st, meta = api.parse_metadata(file)
        items, keep = [], [meta]
        for _ in range(4):
            dev = torch.from_numpy(np.frombuffer(file, dtype=np.uint8).copy()).cuda()
            src = CompressedInput()
            src.bytes = ConstBytes(dev.data_ptr(), len(file))
            src.metadata = meta.handle
            item = BatchItem()
            item.compressed_input = src
            if kind == "fused":
                out = torch.empty(W * H * 4, dtype=torch.uint8, device="cuda")
                item.output = api.view(out, 2, W, H, W * 4)
                item.roi = api.Roi(0, 0, W, H)
                item.calibration.offset.scalar = 100.0
                item.calibration.gain.scalar = 1.05
            else:
                out = torch.empty(W * H * 2, dtype=torch.uint8, device="cuda")
                item.output = api.view(out, 1, W, H, W * 2)
            items.append(item)
            keep += [dev, out]
        op = cuda.Operation.decode_calibrate if kind == "fused" else cuda.Operation.decompress
        st, plan = cuda.prepare_batch(cuda.make_request(op, items), None, stream)
        executor = cuda.decode_calibrate_async if kind == "fused" else cuda.decompress_async
    assert st == Status.success, st
    ws = torch.empty(max(plan.workspace_bytes(), 256), dtype=torch.uint8, device="cuda")
    res = torch.zeros(16 * 4, dtype=torch.uint8, device="cuda")
    for _ in range(launches):
        assert executor(plan, ws, res, stream) == Status.success
    torch.cuda.synchronize()
    recs = res.cpu().numpy().view(np.uint64).reshape(4, 2)
    assert all(int(r[0]) == 0 for r in recs), recs
    print(json.dumps({"profile_case": kind, "launches": launches, "images_per_launch": 4}))


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--profile", choices=["decode", "fused", "encode"], default=None,
                   help="run only a small case for ncu captures and exit")
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3000)
    p.add_argument("--warmup", type=int, default=20)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--copies", type=int, default=4)
    p.add_argument("--cpu-seconds", type=float, default=10.0)
    args = p.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.profile:
        run_profile_case(args.profile)
        return

    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    line, shapes = run_ours(args, rank, world, local, torch, dist)
    if rank == 0:
        line["cpu_baseline"] = cpu_baseline(shapes, args.cpu_seconds)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
