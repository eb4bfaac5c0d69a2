"""Benchmark of the TileStream GPU codec path on B200.

Workload (the config the headline metric is quoted on, fits one GPU): a uint16 4096x4096 detector
frame (seeded synthetic generator, seed 2) encoded with tiles 128x32, 64x64 and 256x16. One step
decodes the three archives device-to-device: one decompress plan over the three, one
decompress_async, one persistent launch. Inputs and outputs rotate
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
import math
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
CYCLE = 20  # steps per replay of the headline's cycle graph (the driver's K)


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, burst copy)"
    return 6650.0, "fallback (6.65 TB/s, earlier measurement on this pool)"


def ncu_traffic():
    """DRAM bytes per headline launch (one step) from the committed ncu summary, when present."""
    path = os.path.join(ROOT, "profiles", "decode_step_3_archives.md")
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
            s["copies"].append({"src": src_dev, "out": out, "plan": plan, "item": item,
                                "input": src})
    # The headline step: one decompress plan over the three archives of a rotation slot (a
    # three-item batch, one persistent launch); the single-archive plans above serve the
    # per-shape figures and the end-to-end path.
    steps = []
    for slot in range(copies):
        st, plan = cuda.prepare_batch(cuda.make_request(
            cuda.Operation.decompress, [s["copies"][slot]["item"] for s in shapes]), None, stream)
        assert st == Status.success, st
        decode_ws = max(decode_ws, plan.workspace_bytes())
        steps.append(plan)
    workspace = torch.empty(max(decode_ws, 256), dtype=torch.uint8, device="cuda")
    results = torch.zeros(16 * 3, dtype=torch.uint8, device="cuda")
    return frame, shapes, steps, workspace, results


def max_over_ranks(value: float, world: int, dist, device: str) -> float:
    """The largest value over the ranks (every rank gets it): the timed region of a multi-GPU
    run lasts as long as its slowest rank."""
    if world == 1:
        return value
    import torch
    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_gbs(bytes_per_step_per_rank: int, steps: int, world: int, ms: float) -> float:
    """Whole-job GB/s: every rank decodes bytes_per_step_per_rank per step (weak scaling)."""
    return bytes_per_step_per_rank * steps * world / (ms / 1e3) / 1e9


def run_ours(args, rank, world, device, torch, dist):
    from tilestream_b200 import api, cuda
    from tilestream_b200.api import Status

    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    copies = args.copies
    frame, shapes, step_plans, workspace, results = prepare_workload(torch, stream, copies)
    wsb = api.MutableBytes(workspace.data_ptr(), workspace.numel())
    recs = [api.ResultBuffer(results.data_ptr() + 16 * k, 1) for k in range(3)]
    step_recs = api.ResultBuffer(results.data_ptr(), 3)

    def enqueue(step):
        st = cuda.decompress_async(step_plans[step % copies], wsb, step_recs, stream)
        assert st == Status.success, st

    # CUDA graphs of the step: one per rotation slot (the decode of that slot's three archives),
    # and cycle graphs holding CYCLE consecutive steps (the slots in rotation order, one graph per
    # starting slot). Inside
    # the cycle the decode kernels are programmatic dependents of one another, as consecutive
    # executions in a stream are, so a step's launch and parsed-payload staging overlap the
    # previous step's end; separate graph launches do not overlap. The executors validate pointers with cudaPointerGetAttributes on the host, which
    # global-mode capture rejects, so capture is relaxed (the validation runs once, at capture).
    graphs, cycles, capture_error = [], None, None
    cycle_steps = copies * max(1, CYCLE // copies)
    try:
        for slot in range(copies):
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=stream, capture_error_mode="relaxed"):
                enqueue(slot)
            graphs.append(g)
        cycles = []
        for start in range(copies):
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=stream, capture_error_mode="relaxed"):
                for k in range(cycle_steps):
                    enqueue((start + k) % copies)
            cycles.append(g)
    except Exception as e:  # noqa: BLE001 - recorded in the JSON line, launches stay eager
        capture_error = str(e).splitlines()[0]
        print(f"graph capture failed, timing eager launches: {capture_error}", file=sys.stderr)
        graphs, cycles = None, None
    torch.cuda.synchronize()

    def replay(i):
        if graphs is not None:
            graphs[i % copies].replay()
        else:
            enqueue(i % copies)

    position = [0]  # the rotation continues across calls: consecutive steps use other slots

    def run_steps(count):
        """count steps: cycle graphs (the one starting at the current slot), then single steps."""
        i = 0
        while cycles is not None and count - i >= cycle_steps:
            cycles[position[0] % copies].replay()
            i += cycle_steps
            position[0] += cycle_steps
        while i < count:
            replay(position[0])
            i += 1
            position[0] += 1

    # Correctness of the benchmarked outputs (one slot per shape).
    for s in shapes:
        s["copies"][0]["out"].zero_()
    enqueue(0)
    torch.cuda.synchronize()
    for s in shapes:
        assert np.array_equal(s["copies"][0]["out"].cpu().numpy().view(np.uint16),
                              frame.reshape(-1)), "decode mismatch"
    r = results.cpu().numpy().view(np.uint64).reshape(3, 2)
    assert all(int(r[k, 0]) == 0 and int(r[k, 1]) == W * H * 2 for k in range(3)), r

    run_steps(args.warmup)
    torch.cuda.synchronize()
    # The timed region is K steps. It is repeated back to back until the repetitions span at
    # least 0.2 s (so that clock samples cover it), each region bracketed by its own events;
    # the reported time is the median region, with the spread beside it.
    pilot0, pilot1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pilot0.record(stream)
    run_steps(args.steps)
    pilot1.record(stream)
    torch.cuda.synchronize()
    pilot_ms = max(pilot0.elapsed_time(pilot1), 1e-3)
    regions = int(min(args.max_regions, max(1, math.ceil(args.min_span_ms / pilot_ms))))
    events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(regions)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(device) as clocks:
        for e0, e1 in events:
            e0.record(stream)
            run_steps(args.steps)
            e1.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    region_ms = sorted(e0.elapsed_time(e1) for e0, e1 in events)
    median_ms = float(np.median(region_ms))
    ms = max_over_ranks(median_ms, world, dist, "cuda")
    step_ms = ms / args.steps
    decoded_per_step = 3 * W * H * 2
    value = aggregate_gbs(decoded_per_step, args.steps, world, ms)
    spread = {"regions": regions, "steps_per_region": args.steps,
              "median_ms": round(median_ms, 5),
              "p05_ms": round(float(np.percentile(region_ms, 5)), 5),
              "p95_ms": round(float(np.percentile(region_ms, 95)), 5),
              "min_ms": round(region_ms[0], 5), "max_ms": round(region_ms[-1], 5),
              "span_ms": round(sum(region_ms), 2)}

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

    # The same step from unparsed files (decode_unparsed_async: the three archives in one launch,
    # index entries, payloads and rows validated on the device), device time per step.
    unparsed_results = torch.zeros(16 * 3, dtype=torch.uint8, device="cuda")

    def unparsed_pass():
        for slot in range(copies):
            entries = [(api.ConstBytes(s["copies"][slot]["src"].data_ptr(), len(s["file"])),
                        s["file"][:64], api.view(s["copies"][slot]["out"], 1, W, H, W * 2))
                       for s in shapes]
            st = cuda.decode_unparsed_async(
                entries, api.ResultBuffer(unparsed_results.data_ptr(), 3), stream)
            assert st == 0, st
    g = None
    if graphs is not None:
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream, capture_error_mode="relaxed"):
            unparsed_pass()
    run_pass = g.replay if g is not None else unparsed_pass
    for _ in range(3):
        run_pass()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(20):
        run_pass()
    e1.record(stream)
    torch.cuda.synchronize()
    unparsed_step_ms = e0.elapsed_time(e1) / (20 * copies)
    recs_u = unparsed_results.cpu().numpy().view(np.uint64).reshape(-1, 2)
    assert all(int(r[0]) == 0 and int(r[1]) == W * H * 2 for r in recs_u), recs_u

    peak, peak_src = measured_peaks()
    alg_per_launch = sum(s["algorithmic"] for s in shapes) # one launch per step
    unparsed = {"workload": "the headline step from unparsed files: the three archives in one "
                            "decode_unparsed_async launch (a result-record clear and the decode), "
                            "validation on the device",
                "step_us": round(unparsed_step_ms * 1e3, 2),
                "decoded_gbs": round(decoded_per_step / unparsed_step_ms / 1e6, 1),
                "roofline_frac": round(alg_per_launch / (unparsed_step_ms / 1e3) / 1e9 / peak, 4),
                "cuda_graph": g is not None}
    launch_ms = step_ms
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
        "gpu_launches": args.steps,
        "timing": spread,
        "cuda_graph": graphs is not None,
        "graph_steps": cycle_steps if cycles is not None else 1,
        **({"graph_capture_error": capture_error} if capture_error else {}),
        "per_shape": per_shape,
        "unparsed_decode": unparsed,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                     "peak_source": peak_src, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "algorithmic_bytes_per_launch": int(alg_per_launch),
                     "traffic": ncu_traffic(),
                     "traffic_source": "copied from the committed ncu capture of the same launch "
                                       "(profiles/decode_step_3_archives.md), not measured here",
                     "kernel": "decode_kernel"},
        "e2e": e2e,
        "clocks": clocks.report(),
    }
    return line, shapes


def run_e2e(args, torch, stream, shapes, wsb, recs):
    """Per step: H2D copy of the three archives from pinned memory, three decodes, D2H copy of
    the three decoded frames into pinned memory. Each archive alternates between two of its
    device copies (each with its own plan, input and output buffers): its H2D copies run on
    one stream and its decodes and D2H copies on another, ordered by events, so the host link
    carries step i + 1's archives while step i's pixels go D2H; the timed region spans all the
    streams."""
    from tilestream_b200 import api, cuda
    pinned_in = [torch.from_numpy(np.frombuffer(s["file"], dtype=np.uint8).copy()).pin_memory()
                 for s in shapes]
    pinned_out = [torch.empty(W * H * 2, dtype=torch.uint8).pin_memory() for _ in shapes]
    n = len(shapes)
    h2d_streams = [torch.cuda.Stream() for _ in shapes]
    streams = [torch.cuda.Stream() for _ in shapes]
    copied = [[torch.cuda.Event() for _ in range(2)] for _ in shapes]
    decoded = [[torch.cuda.Event() for _ in range(2)] for _ in shapes]
    results = torch.zeros(16 * n, dtype=torch.uint8, device="cuda")
    own = [api.ResultBuffer(results.data_ptr() + 16 * k, 1) for k in range(n)]
    # Each workspace is used by one stream's decodes only.
    spaces = [torch.empty(wsb.size, dtype=torch.uint8, device="cuda") for _ in shapes]
    steps = max(3, min(args.steps, 50))
    counter = [0]

    def step(decode=True):
        i = counter[0]
        counter[0] += 1
        slot = i % 2
        for k, s in enumerate(shapes):
            c = s["copies"][slot]
            h, st_k = h2d_streams[k], streams[k]
            if i >= 2:
                h.wait_event(decoded[k][slot])  # the decode of step i - 2 has read this input
            with torch.cuda.stream(h):
                c["src"][:len(s["file"])].copy_(pinned_in[k], non_blocking=True)
            copied[k][slot].record(h)
            st_k.wait_event(copied[k][slot])
            if decode:
                ws = api.MutableBytes(spaces[k].data_ptr(), spaces[k].numel())
                st = cuda.decompress_async(c["plan"], ws, own[k], st_k)
                assert st == 0, st
            decoded[k][slot].record(st_k)
            with torch.cuda.stream(st_k):
                pinned_out[k].copy_(c["out"], non_blocking=True)

    def timed(count, decode=True):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for st in streams + h2d_streams:
            st.wait_event(e0)
        for _ in range(count):
            step(decode)
        for st in streams + h2d_streams:
            stream.wait_stream(st)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    timed(4)
    ms = timed(steps)
    # The host link's ceiling on this box: the same copies, streams and events, no decode.
    timed(4, decode=False)
    link_ms = timed(steps, decode=False)
    timed(2)  # leaves decoded outputs in the last slot for the check below
    recs_host = results.cpu().numpy().view(np.uint64).reshape(-1, 2)
    assert all(int(r[0]) == 0 and int(r[1]) == W * H * 2 for r in recs_host), recs_host
    last = (counter[0] - 1) % 2
    for k, s in enumerate(shapes):
        assert torch.equal(pinned_out[k], s["copies"][last]["out"].cpu())
    h2d = sum(len(s["file"]) for s in shapes)
    d2h = n * W * H * 2

    # From the file: every step starts from each archive's .tsc bytes in pinned host memory and
    # runs parse_metadata (the library's host parser) and prepare_batch (a new plan) for it on
    # the host, then the same copies and decode. The host parses and prepares step i + 1 while
    # the GPU copies and decodes step i; a plan is released once the decode that used it has
    # completed (two steps later, the slot's reuse).
    prep_streams = [torch.cuda.Stream() for _ in shapes]
    held = [[None, None] for _ in shapes]
    fcounter = [0]
    host_ms = {"parse": [], "prepare": []}
    import concurrent.futures as cf
    pool = cf.ThreadPoolExecutor(max_workers=n)

    def make_plan(k, i):
        """Archive k's parse and plan for step i, on a worker thread (the library's host calls
        release the interpreter lock). The slot's previous plan is released once the decode that
        used it has completed."""
        slot = i % 2
        s, c = shapes[k], shapes[k]["copies"][slot]
        if held[k][slot] is not None:
            held[k][slot][2].synchronize()
            held[k][slot] = None
        t0 = time.perf_counter()
        st, meta = api.parse_metadata(pinned_in[k].numpy(), size=len(s["file"]))
        assert st == 0, st
        t1 = time.perf_counter()
        src = api.CompressedInput()
        src.bytes = api.ConstBytes(c["src"].data_ptr(), len(s["file"]))
        src.metadata = meta.handle
        item = api.BatchItem()
        item.compressed_input = src
        item.output = api.view(c["out"], 1, W, H, W * 2)
        st, plan = cuda.prepare_batch(cuda.make_request(cuda.Operation.decompress, [item]),
                                      None, prep_streams[k])
        assert st == 0, st
        host_ms["parse"].append((t1 - t0) * 1e3)
        host_ms["prepare"].append((time.perf_counter() - t1) * 1e3)
        return meta, plan

    pending = {}

    def submit(i):
        pending[i] = [pool.submit(make_plan, k, i) for k in range(n)]

    def step_file():
        i = fcounter[0]
        fcounter[0] += 1
        slot = i % 2
        if i not in pending:
            submit(i)
        made = [f.result() for f in pending.pop(i)]
        for k, s in enumerate(shapes):
            c = s["copies"][slot]
            meta, plan = made[k]
            h, st_k = h2d_streams[k], streams[k]
            if i >= 2:
                h.wait_event(decoded[k][slot])
            with torch.cuda.stream(h):
                c["src"][:len(s["file"])].copy_(pinned_in[k], non_blocking=True)
            copied[k][slot].record(h)
            st_k.wait_event(copied[k][slot])
            ws = api.MutableBytes(spaces[k].data_ptr(), spaces[k].numel())
            assert cuda.decompress_async(plan, ws, own[k], st_k) == 0
            done = torch.cuda.Event()
            done.record(st_k)
            decoded[k][slot].record(st_k)
            held[k][slot] = (meta, plan, done)
            with torch.cuda.stream(st_k):
                pinned_out[k].copy_(c["out"], non_blocking=True)
        submit(i + 1)  # the next step's parses and plans, while this step runs on the GPU

    def timed_file(count):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for st in streams + h2d_streams:
            st.wait_event(e0)
        for _ in range(count):
            step_file()
        for st in streams + h2d_streams:
            stream.wait_stream(st)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    timed_file(4)
    host_ms["parse"].clear()
    host_ms["prepare"].clear()
    file_ms = timed_file(steps)
    torch.cuda.synchronize()
    for futures in pending.values():
        for f in futures:
            f.result()
    pool.shutdown()
    held.clear()
    recs_host = results.cpu().numpy().view(np.uint64).reshape(-1, 2)
    assert all(int(r[0]) == 0 and int(r[1]) == W * H * 2 for r in recs_host), recs_host
    last = (fcounter[0] - 1) % 2
    for k, s in enumerate(shapes):
        assert torch.equal(pinned_out[k], s["copies"][last]["out"].cpu())
    from_file = {"value": round(n * W * H * 2 * steps / (file_ms / 1e3) / 1e9, 2), "unit": "GB/s",
                 "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": steps,
                 "ms_per_step": round(file_ms / steps, 4),
                 "host_work": "parse_metadata + prepare_batch of every archive, every step, "
                              f"on {n} host threads one step ahead of the GPU",
                 "host_ms_per_archive": {k: round(float(np.mean(v)), 3) if v else None
                                         for k, v in host_ms.items()}}
    # From the file, validated on the device: every step starts from each archive's .tsc bytes
    # in pinned host memory; the host checks the file's 64-byte header (read from the pinned
    # file), the H2D copy brings the file to the device, and decode_unparsed_async validates
    # every index entry, payload and row descriptor there with parse_metadata's rules while it
    # decodes; then the D2H copy of the pixels. No host parse, no plan.
    unparsed_results = torch.zeros(16 * n, dtype=torch.uint8, device="cuda")
    ucounter = [0]

    def step_unparsed():
        i = ucounter[0]
        ucounter[0] += 1
        slot = i % 2
        for k, s in enumerate(shapes):
            c = s["copies"][slot]
            h, st_k = h2d_streams[k], streams[k]
            header = pinned_in[k][:64].numpy().tobytes()
            if i >= 2:
                h.wait_event(decoded[k][slot])
            with torch.cuda.stream(h):
                c["src"][:len(s["file"])].copy_(pinned_in[k], non_blocking=True)
            copied[k][slot].record(h)
            st_k.wait_event(copied[k][slot])
            entry = (api.ConstBytes(c["src"].data_ptr(), len(s["file"])), header,
                     api.view(c["out"], 1, W, H, W * 2))
            st = cuda.decode_unparsed_async(
                [entry], api.ResultBuffer(unparsed_results.data_ptr() + 16 * k, 1), st_k)
            assert st == 0, st
            decoded[k][slot].record(st_k)
            with torch.cuda.stream(st_k):
                pinned_out[k].copy_(c["out"], non_blocking=True)

    def timed_unparsed(count):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for st in streams + h2d_streams:
            st.wait_event(e0)
        for _ in range(count):
            step_unparsed()
        for st in streams + h2d_streams:
            stream.wait_stream(st)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    # The pixels of the host-parsed leg (checked above) are the reference for this leg's last
    # step; the device outputs are cleared first.
    want = [p.clone() for p in pinned_out]
    for k, s in enumerate(shapes):
        s["copies"][0]["out"].zero_()
        s["copies"][1]["out"].zero_()
    torch.cuda.synchronize()
    timed_unparsed(4)
    unparsed_ms = timed_unparsed(steps)
    recs_host = unparsed_results.cpu().numpy().view(np.uint64).reshape(-1, 2)
    assert all(int(r[0]) == 0 and int(r[1]) == W * H * 2 for r in recs_host), recs_host
    for k in range(n):
        assert torch.equal(pinned_out[k], want[k])
    device_validated = {
        "value": round(n * W * H * 2 * steps / (unparsed_ms / 1e3) / 1e9, 2), "unit": "GB/s",
        "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": steps,
        "ms_per_step": round(unparsed_ms / steps, 4),
        "host_work": "header check of every archive, every step (decode_unparsed_async); index "
                     "entries, payloads and rows validated on the device with parse_metadata's "
                     "rules"}

    resident = {"value": round(n * W * H * 2 * steps / (ms / 1e3) / 1e9, 2), "unit": "GB/s",
            "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": steps,
            "ms_per_step": round(ms / steps, 4), "streams": 2 * n,
            "buffers": "two device copies per archive, alternating",
            "copies_only_ms_per_step": round(link_ms / steps, 4),
            "link_frac": round(link_ms / ms, 4)}
    # The headline e2e is like-for-like with the reference arm, whose cpu::decompress validates
    # every file on every decode: each step starts from the file's bytes and validates all of
    # them, on the device. The host-parse and resident-plan figures stand beside it.
    return {**device_validated, "host_parsed": from_file, "resident_plans": resident}


def best_ms(fn, reps: int = 10) -> float:
    best = float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        best = min(best, time.perf_counter() - t0)
    return best * 1e3


def host_parse(shapes):
    """parse_metadata of the three archives through the product API (best of 10 each)."""
    from tilestream_b200 import api
    out = {}
    for s in shapes:
        src = np.frombuffer(s["file"], dtype=np.uint8)
        out["%dx%d" % s["tile"]] = round(best_ms(lambda: api.parse_metadata(src)), 3)
    return {"unit": "ms per 4096x4096 archive (20 MB, 4096 tiles)", "ms": out,
            "threads": min(8, os.cpu_count() or 1)}


def cpu_baseline(shapes, seconds):
    import oracle
    archive = shapes[0]["file"]
    ref = oracle.Reference.available()
    threads = os.cpu_count() or 1
    rate, images = cpu_decode_rate(archive, seconds, threads, ref)
    line = {"value": round(rate / 1e9, 3), "unit": "GB/s", "cores": threads,
            "kind": "reference" if ref else "port",
            "sample": f"{images} decodes of the 4096x4096 uint16 128x32 archive, one image per "
                      f"thread, {seconds:.0f} s"}
    one, images1 = cpu_decode_rate(archive, max(1.0, seconds / 5), 1, ref)
    line["single_thread"] = {"value": round(one / 1e9, 3), "unit": "GB/s",
                             "sample": f"{images1} decodes on one thread"}
    if ref:
        codec = oracle.Reference()
        line["parse_ms"] = {"%dx%d" % s["tile"]: round(best_ms(
            lambda s=s: codec.parse_status(s["file"])), 3) for s in shapes}
    return line


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
        "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": args.gpus,
        "device": "host CPU cores (the reference codec has no GPU path to call here)",
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


def encode_on_gpu(torch, stream, inputs, ptype, tile):
    """Encodes device images of one pixel type with one compress plan (tile geometry `tile`).
    inputs: list of (flat uint8 device tensor, width, height, pitch). Returns the .tsc files as
    host bytes (the plan-based GPU encoder, byte-identical to the CPU codec per the tests)."""
    from tilestream_b200 import api, cuda
    from tilestream_b200.api import BatchItem, Status, TileShape
    items, outs = [], []
    for dev, w, h, pitch in inputs:
        st, bound = api.compress_bound(api.image_spec(ptype, w, h), TileShape(*tile))
        out = torch.empty(bound, dtype=torch.uint8, device="cuda")
        item = BatchItem()
        item.input = api.const_view(dev, ptype, w, h, pitch, dev.numel())
        item.compressed_output = api.MutableBytes(out.data_ptr(), bound)
        items.append(item)
        outs.append(out)
    st, plan = cuda.prepare_batch(cuda.make_request(cuda.Operation.compress, items,
                                                    TileShape(*tile)), None, stream)
    assert st == Status.success, st
    ws = torch.empty(max(plan.workspace_bytes(), 256), dtype=torch.uint8, device="cuda")
    res = torch.zeros(16 * len(items), dtype=torch.uint8, device="cuda")
    assert cuda.compress_async(plan, ws, res, stream) == Status.success
    torch.cuda.synchronize()
    sizes = res.cpu().numpy().view(np.uint64).reshape(-1, 2)[:, 1]
    return [out[:int(n)].cpu().numpy().tobytes() for out, n in zip(outs, sizes)]


def time_graph(torch, stream, fn, steps, warmup):
    """Captures fn (which enqueues on stream) as a CUDA graph; returns ms per replay."""
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream, capture_error_mode="relaxed"):
        fn()
    for _ in range(warmup):
        g.replay()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        g.replay()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def calibration_contract(x, offset, gain, result) -> dict:
    """Checks binary32 calibration results against the reference's numerical contract
    (tests/numerics/support.h: bounds 45-57, expected classes 119-142, checks 181-226). Each
    calibration is classed from its inputs and the FP64 reference (x - offset) * gain: NaN
    input, invalid, infinite, intermediate overflow (the difference overflows), overflow, zero,
    subnormal or normal. The result must then be a NaN; an infinity of the reference's sign;
    the IEEE product of the rounded difference; an infinity, or FLT_MAX at the threshold, of
    the reference's sign; a zero of its sign; within 2^-149 (subnormal); or within 1.5 ulp and
    2^-23 relative (normal). All arguments are float32 arrays of one shape (offset and gain may
    be scalars). Returns the count per class, the violations and the largest normal-class
    error in ulp."""
    x = np.asarray(x, np.float32).ravel()
    r = np.asarray(result, np.float32).ravel()
    o = np.broadcast_to(np.asarray(offset, np.float32).ravel(), x.shape)
    g = np.broadcast_to(np.asarray(gain, np.float32).ravel(), x.shape)
    threshold = 2.0 ** 128 - 2.0 ** 103  # smallest magnitude that rounds to infinity
    with np.errstate(all="ignore"):
        difference = x.astype(np.float64) - o
        ref = difference * g
        mag = np.abs(ref)
        nan_input = np.isnan(x) | np.isnan(o) | np.isnan(g)
        invalid = ~nan_input & np.isnan(ref)
        infinite = ~nan_input & ~invalid & np.isinf(ref)
        rest = ~(nan_input | invalid | infinite)
        intermediate = rest & (np.abs(difference) >= threshold)
        rest &= ~intermediate
        overflow = rest & (mag >= threshold)
        rest &= ~overflow
        zero = rest & (mag == 0)
        subnormal = rest & ~zero & (mag < 2.0 ** -126)
        normal = rest & ~zero & ~subnormal
        sign = np.signbit(r) == np.signbit(ref)
        ieee = ((x - o).astype(np.float32) * g).astype(np.float32)
        same = (r.view(np.uint32) == ieee.view(np.uint32)) | (np.isnan(r) & np.isnan(ieee))
        err = np.abs(r.astype(np.float64) - ref)
        _, exponent = np.frexp(mag)
        ulp = np.where(mag < 2.0 ** -126, 2.0 ** -149, np.ldexp(1.0, exponent - 24))
        ulps = err / ulp
        relative = err / np.maximum(mag, 2.0 ** -126)
        flt_max = float(np.finfo(np.float32).max)
        ok = np.select(
            [nan_input | invalid, infinite, intermediate, overflow, zero, subnormal],
            [np.isnan(r), np.isinf(r) & sign, same,
             sign & (np.isinf(r) | ((np.abs(r) == flt_max) &
                                    (mag < threshold * (1 + 2.0 ** -24)))),
             (r == 0) & sign,
             np.isfinite(r) & ~((r == 0) & ~sign) & (err <= 2.0 ** -149 * (1 + 2.0 ** -20))],
            np.where(np.isinf(r), sign & (mag * (1 + 2.0 ** -24) >= threshold),
                     ~np.isnan(r) & (ulps <= 1.5 + 2.0 ** -20) &
                     (relative <= 2.0 ** -23 * (1 + 2.0 ** -20))))
    finite_normal = normal & np.isfinite(r)
    classes = {"nan_input": nan_input, "invalid": invalid, "infinite": infinite,
               "intermediate_overflow": intermediate, "overflow": overflow, "zero": zero,
               "subnormal": subnormal, "normal": normal}
    return {"classes": {k: int(v.sum()) for k, v in classes.items()},
            "violations": int((~ok).sum()),
            "max_ulp_normal": float(ulps[finite_normal].max()) if finite_normal.any() else 0.0}


def merge_contract(total: dict | None, part: dict) -> dict:
    if total is None:
        return part
    return {"classes": {k: total["classes"][k] + part["classes"][k] for k in total["classes"]},
            "violations": total["violations"] + part["violations"],
            "max_ulp_normal": max(total["max_ulp_normal"], part["max_ulp_normal"])}


def run_calibrated(args, torch, stream, peak):
    """Config 3: float32 4096x4096 smooth field with special words, fused decode + calibration
    with per-pixel FP32 offset ~ N(100, 5) and gain ~ U(0.9, 1.1) maps."""
    from tilestream_b200 import api, cuda, workloads
    from tilestream_b200.api import BatchItem, CompressedInput, ConstBytes, Status
    frame = workloads.field_frame(W, H, seed=3)
    offset, gain = workloads.calibration_maps(W, H, seed=5)
    dev_frame = torch.from_numpy(frame.view(np.uint8).reshape(-1).copy()).cuda()
    file = encode_on_gpu(torch, stream, [(dev_frame, W, H, W * 4)], 2, (128, 32))[0]
    st, meta = api.parse_metadata(file)
    assert st == Status.success
    dev_off = torch.from_numpy(offset.view(np.uint8).reshape(-1).copy()).cuda()
    dev_gain = torch.from_numpy(gain.view(np.uint8).reshape(-1).copy()).cuda()
    copies = []
    for _ in range(2):
        src_dev = torch.from_numpy(np.frombuffer(file, dtype=np.uint8).copy()).cuda()
        out = torch.empty(W * H * 4, dtype=torch.uint8, device="cuda")
        plain = torch.empty(W * H * 4, dtype=torch.uint8, device="cuda")
        src = CompressedInput()
        src.bytes = ConstBytes(src_dev.data_ptr(), len(file))
        src.metadata = meta.handle
        item = BatchItem()
        item.compressed_input = src
        item.output = api.view(out, 2, W, H, W * 4)
        item.roi = api.Roi(0, 0, W, H)
        item.calibration.offset.kind = cuda.ParameterKind.map
        item.calibration.offset.map = api.const_view(dev_off, 2, W, H, W * 4)
        item.calibration.gain.kind = cuda.ParameterKind.map
        item.calibration.gain.map = api.const_view(dev_gain, 2, W, H, W * 4)
        st, plan = cuda.prepare_batch(cuda.make_request(cuda.Operation.decode_calibrate, [item]),
                                      None, stream)
        assert st == Status.success, st
        pitem = BatchItem()
        pitem.compressed_input = src
        pitem.output = api.view(plain, 2, W, H, W * 4)
        st, pplan = cuda.prepare_batch(cuda.make_request(cuda.Operation.decompress, [pitem]),
                                       None, stream)
        assert st == Status.success, st
        copies.append({"src": src_dev, "out": out, "plan": plan, "plain": plain, "pplan": pplan})
    ws = torch.empty(max(copies[0]["plan"].workspace_bytes(), 256), dtype=torch.uint8,
                     device="cuda")
    res = torch.zeros(16, dtype=torch.uint8, device="cuda")
    c = copies[0]
    assert cuda.decompress_async(c["pplan"], ws, res, stream) == Status.success
    assert cuda.decode_calibrate_async(c["plan"], ws, res, stream) == Status.success
    torch.cuda.synchronize()
    words = c["plain"].cpu().numpy().view(np.uint32)
    exact = bool(np.array_equal(words, frame.reshape(-1)))
    got = c["out"].cpu().numpy().view(np.float32)
    x = frame.reshape(-1).view(np.float32)
    with np.errstate(all="ignore"):
        host_form = ((x - offset.reshape(-1)).astype(np.float32) * gain.reshape(-1)).astype(
            np.float32)
        ref = (x.astype(np.float64) - offset.reshape(-1).astype(np.float64)) * \
            gain.reshape(-1).astype(np.float64)
    same = (got.view(np.uint32) == host_form.view(np.uint32)) | (np.isnan(got) &
                                                                 np.isnan(host_form))
    normal = np.isfinite(ref) & (np.abs(ref) >= 2.0 ** -126) & np.isfinite(got)
    ulp = np.spacing(np.abs(ref[normal]).astype(np.float32)).astype(np.float64)
    max_ulp = float(np.max(np.abs(got[normal].astype(np.float64) - ref[normal]) / ulp))
    contract = calibration_contract(x, offset, gain, got)

    def step(k=[0]):
        cc = copies[k[0] % 2]
        k[0] += 1
        cuda.decode_calibrate_async(cc["plan"], ws, res, stream)

    def both():
        for cc in copies:
            cuda.decode_calibrate_async(cc["plan"], ws, res, stream)

    ms = time_graph(torch, stream, both, max(3, args.steps // 100), args.warmup) / 2

    # Standalone calibration of the decoded words with the same maps (streaming kernel): 16 B
    # per pixel (FP32 in, two FP32 maps, FP32 out), 268 MB per launch, more than the L2 holds.
    cal_out = torch.empty(W * H * 4, dtype=torch.uint8, device="cuda")
    citem = BatchItem()
    citem.input = api.const_view(c["plain"], 2, W, H, W * 4)
    citem.output = api.view(cal_out, 2, W, H, W * 4)
    citem.calibration.offset.kind = cuda.ParameterKind.map
    citem.calibration.offset.map = api.const_view(dev_off, 2, W, H, W * 4)
    citem.calibration.gain.kind = cuda.ParameterKind.map
    citem.calibration.gain.map = api.const_view(dev_gain, 2, W, H, W * 4)
    st, cplan = cuda.prepare_batch(cuda.make_request(cuda.Operation.calibrate, [citem]), None,
                                   stream)
    assert st == Status.success, st
    assert cuda.calibrate_async(cplan, None, res, stream) == Status.success
    torch.cuda.synchronize()
    standalone_same = bool(torch.equal(cal_out, c["out"]))  # fused == standalone, bit for bit
    cal_ms = time_graph(torch, stream, lambda: cuda.calibrate_async(cplan, None, res, stream),
                        max(3, args.steps // 100), args.warmup)
    cal_alg = W * H * 4 * 4

    tiles = meta.tiles
    alg = int(tiles["length"].sum()) + 32 * len(tiles) + W * H * 4 * 3  # output + 2 maps
    return {"workload": "float32 4096x4096 field (seed 3), 0.1% special words, fused decode + "
                        "calibration with FP32 offset and gain maps, tiles 128x32",
            "launch_us": round(ms * 1e3, 2),
            "calibrated_gbs": round(W * H * 4 / ms / 1e6, 1),
            "roofline": {"achieved": round(alg / ms / 1e6, 1), "peak": peak,
                         "frac": round(alg / ms / 1e6 / peak, 4), "unit": "GB/s",
                         "algorithmic_bytes_per_launch": alg},
            "pixels_bit_exact_before_calibration": exact,
            "calibrated_equals_host_two_rounding_form": bool(np.all(same)),
            "max_ulp_vs_fp64_normal_results": round(max_ulp, 4),
            "ulp_bound": 1.5,
            "contract": contract,
            "standalone_calibrate": {
                "workload": "the decoded field calibrated with the same FP32 maps",
                "launch_us": round(cal_ms * 1e3, 2),
                "roofline": {"achieved": round(cal_alg / cal_ms / 1e6, 1), "peak": peak,
                             "frac": round(cal_alg / cal_ms / 1e6 / peak, 4), "unit": "GB/s",
                             "algorithmic_bytes_per_launch": cal_alg},
                "equals_fused_bit_for_bit": standalone_same}}


def run_archive_roi(args, torch, shapes):
    """ROIs of archives held in pinned host memory, decoded with calibration into FP32 on the
    device (the reference benchmark's archive ROI mode, benchmarks/codec_benchmark.cpp:153-320).
    Per request: the ROI's tile payloads are copied to the device on a copy stream, a plan is
    prepared on its own stream, and decode_calibrate runs on a compute stream after the copy's
    event; requests pipeline (the host enqueues request k + 1 while the device works on k).
    Three ways to get the payloads to the device are timed: `direct` (stage_roi_tiles: one copy
    per tile row straight from the pinned archive), `gather` (the reference's way: host copies
    of the ROI's tiles into a pinned staging buffer, then one copy) and `whole_archive` (the
    whole file copied per request). `direct_batched` stages the same way but decodes the 64
    requests as one mixed batch (one plan and one launch for all of them: throughput, with the
    batch's latency for every request). Decoded bytes count ROI pixels at 2 B (the stored
    type)."""
    from tilestream_b200 import api, cuda
    from tilestream_b200.api import (BatchItem, Calibration, CompressedInput, ConstBytes,
                                     MutableBytes, Roi, Status, TileMapping)
    rng = np.random.default_rng(17)
    n = 64
    pinned = [torch.from_numpy(np.frombuffer(s["file"], dtype=np.uint8).copy()).pin_memory()
              for s in shapes]
    reqs = []
    for k in range(n):
        a = k % len(shapes)
        w = int(np.exp(rng.uniform(np.log(128), np.log(2048))))
        h = int(np.exp(rng.uniform(np.log(128), np.log(2048))))
        x, y = int(rng.integers(0, W - w + 1)), int(rng.integers(0, H - h + 1))
        reqs.append((a, (x, y, w, h)))
    copy, prep, compute = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    slots = []
    for a, roi in reqs:
        meta = shapes[a]["meta"]
        st, need = cuda.roi_staging_size(meta, Roi(*roi))
        assert st == Status.success
        slots.append({
            "need": need, "staging": torch.empty(need.bytes, dtype=torch.uint8, device="cuda"),
            "host_staging": torch.empty(need.bytes, dtype=torch.uint8).pin_memory(),
            "maps": (TileMapping * need.tiles)(),
            "out": torch.empty(roi[2] * roi[3] * 4, dtype=torch.uint8, device="cuda"),
            # the whole-archive way: a device copy of the archive per request
            "archive": torch.empty(len(shapes[a]["file"]), dtype=torch.uint8, device="cuda"),
            "event": torch.cuda.Event()})
    results = torch.zeros(16 * n, dtype=torch.uint8, device="cuda")
    cal = Calibration()
    cal.offset.scalar = 100.0
    cal.gain.scalar = 1.05

    # The gather's copies, one per tile row of the ROI (its tiles are adjacent in the file),
    # and its mappings: worked out once, like the reference's tile lists, and not timed.
    for i, (a, roi) in enumerate(reqs):
        s = slots[i]
        tiles = shapes[a]["meta"].tiles
        tw, th = shapes[a]["tile"]
        across = -(-W // tw)
        x, y, w, h = roi
        runs, maps, at = [], [], 0
        for r in range(y // th, (y + h - 1) // th + 1):
            first, last = r * across + x // tw, r * across + (x + w - 1) // tw
            b = int(tiles["offset"][first])
            e = int(tiles["offset"][last]) + int(tiles["length"][last])
            runs.append((b, e, at))
            maps += [TileMapping(t, at + int(tiles["offset"][t]) - b)
                     for t in range(first, last + 1)]
            at += e - b
        s["gruns"], s["gbytes"] = runs, at
        s["gmaps"] = (TileMapping * len(maps))(*maps)

    def item_for(i, mode):
        a, roi = reqs[i]
        s = slots[i]
        src = CompressedInput()
        src.metadata = shapes[a]["meta"].handle
        if mode == "whole_archive":
            src.bytes = ConstBytes(s["archive"].data_ptr(), len(shapes[a]["file"]))
        elif mode == "gather":
            src.bytes = ConstBytes(s["staging"].data_ptr(), s["gbytes"])
            src.mappings = s["gmaps"]
            src.mapping_count = s["need"].tiles
        else:
            src.bytes = ConstBytes(s["staging"].data_ptr(), s["need"].bytes)
            src.mappings = s["maps"]
            src.mapping_count = s["need"].tiles
        it = BatchItem()
        it.compressed_input = src
        it.output = api.view(s["out"], 2, roi[2], roi[3], roi[2] * 4, s["out"].numel())
        it.roi = Roi(*roi)
        it.calibration = cal
        return it

    def gather(i):
        """The reference's host gather: the ROI's tiles, row by row, into pinned staging."""
        a, _ = reqs[i]
        s = slots[i]
        src = pinned[a].numpy()
        dst = s["host_staging"].numpy()
        for b, e, at in s["gruns"]:
            dst[at:at + e - b] = src[b:e]

    host_us = {"stage": 0.0, "prepare": 0.0, "launch": 0.0}

    def step_batched():
        """All the batch's ROIs staged on the copy stream, then one mixed batch of their 64
        decode_calibrate items (one plan, one launch) after the copies' event."""
        for i, (a, roi) in enumerate(reqs):
            s = slots[i]
            st, _ = cuda.stage_roi_tiles(
                shapes[a]["meta"], Roi(*roi), ConstBytes(pinned[a].data_ptr(),
                                                         len(shapes[a]["file"])),
                MutableBytes(s["staging"].data_ptr(), s["need"].bytes), s["maps"], copy)
            assert st == Status.success, st
        staged = torch.cuda.Event()
        staged.record(copy)
        items = [(cuda.Operation.decode_calibrate, item_for(i, "direct")) for i in range(n)]
        st, batch = cuda.prepare_mixed_batch(items, results, prep, graph=False)
        assert st == Status.success, st
        compute.wait_event(staged)
        assert batch.run(compute) == Status.success
        compute.synchronize()
        copy.synchronize()
        return [batch]

    def step(mode):
        if mode == "direct_batched":
            return step_batched()
        plans = []
        for i, (a, roi) in enumerate(reqs):
            s = slots[i]
            t0 = time.perf_counter()
            if mode == "direct":
                st, _ = cuda.stage_roi_tiles(
                    shapes[a]["meta"], Roi(*roi), ConstBytes(pinned[a].data_ptr(),
                                                             len(shapes[a]["file"])),
                    MutableBytes(s["staging"].data_ptr(), s["need"].bytes), s["maps"], copy)
                assert st == Status.success, st
            elif mode == "gather":
                gather(i)
                with torch.cuda.stream(copy):
                    s["staging"][:s["gbytes"]].copy_(s["host_staging"][:s["gbytes"]],
                                                     non_blocking=True)
            else:
                with torch.cuda.stream(copy):
                    s["archive"].copy_(pinned[a], non_blocking=True)
            s["event"].record(copy)
            t1 = time.perf_counter()
            st, plan = cuda.prepare_batch(cuda.make_request(
                cuda.Operation.decode_calibrate, [item_for(i, mode)]), None, prep)
            assert st == Status.success, st
            assert plan.workspace_bytes() <= ws.numel()
            plans.append(plan)
            t2 = time.perf_counter()
            compute.wait_event(s["event"])
            rb = api.ResultBuffer(results.data_ptr() + 16 * i, 1)
            assert cuda.decode_calibrate_async(plan, MutableBytes(ws.data_ptr(), ws.numel()), rb,
                                               compute) == Status.success
            t3 = time.perf_counter()
            if mode == "direct":
                host_us["stage"] += (t1 - t0) * 1e6
                host_us["prepare"] += (t2 - t1) * 1e6
                host_us["launch"] += (t3 - t2) * 1e6
        compute.synchronize()
        copy.synchronize()
        return plans

    need_ws = 256
    for i in range(n):
        for mode in ("gather", "whole_archive"):
            st, plan = cuda.prepare_batch(cuda.make_request(cuda.Operation.decode_calibrate,
                                                            [item_for(i, mode)]), None, prep)
            assert st == Status.success, st
            need_ws = max(need_ws, plan.workspace_bytes())
    ws = torch.empty(need_ws, dtype=torch.uint8, device="cuda")
    px = sum(r[1][2] * r[1][3] for r in reqs)
    out = {"workload": f"{n} ROIs of the three 4096x4096 uint16 archives in pinned host memory, "
                       "sides log-uniform 128..2048, decode_calibrate to FP32 (offset 100.0, "
                       "gain 1.05), one plan per request",
           "mean_roi_mpx": round(px / n / 1e6, 3)}
    for mode in ("direct", "direct_batched", "gather", "whole_archive"):
        step(mode)
        for k in host_us:
            host_us[k] = 0.0
        times = []
        for _ in range(5):
            t0 = time.perf_counter()
            step(mode)
            times.append(time.perf_counter() - t0)
        sec = statistics.median(times)
        recs = results.cpu().numpy().view(np.uint64).reshape(-1, 2)
        assert all(int(r[0]) == 0 for r in recs), recs[:4]
        h2d = {"direct": sum(s["need"].bytes for s in slots),
               "direct_batched": sum(s["need"].bytes for s in slots),
               "gather": sum(s["gbytes"] for s in slots),
               "whole_archive": sum(len(shapes[a]["file"]) for a, _ in reqs)}[mode]
        out[mode] = {"ms_per_batch": round(sec * 1e3, 3), "requests_per_s": round(n / sec, 1),
                     "decoded_gbs": round(px * 2 / sec / 1e9, 2),
                     "h2d_mb_per_batch": round(h2d / 1e6, 2)}
        if mode == "direct":
            out[mode]["host_us_per_request"] = {k: round(v / (5 * n), 1)
                                                for k, v in host_us.items()}
    # The outputs of the last (whole-archive) pass against a direct-staged pass.
    keep = [s["out"].clone() for s in slots]
    step("direct")
    assert all(torch.equal(k, s["out"]) for k, s in zip(keep, slots)), "staged != resident"
    out["copies_per_request"] = {
        "direct": round(statistics.mean(s["need"].copies for s in slots), 1),
        "gather": round(statistics.mean(len(s["gruns"]) for s in slots), 1)}
    return out


def mixed_archives(torch, stream, n):
    """The archives of config 4: n archives with width and height uniform in 257..4096, 70%
    uint16 / 30% float32, a random tile geometry each (seed 4), encoded on the GPU and resident
    in device memory, each with a whole-image decode item into pitched rows and its own
    single-image plan. Returns (entries, plans, frames, keep, decoded_bytes, algorithmic
    bytes)."""
    from tilestream_b200 import api, cuda, workloads
    from tilestream_b200.api import BatchItem, CompressedInput, ConstBytes, Status
    rng = np.random.default_rng(4)
    dims = rng.integers(257, 4097, size=(n, 2))
    types = np.where(rng.random(n) < 0.7, 1, 2)
    shapes = [SHAPES[i] for i in rng.integers(0, 3, n)]
    frames = []
    for k in range(n):
        w, h = int(dims[k, 0]), int(dims[k, 1])
        if types[k] == 1:
            f = workloads.detector_frame_torch(w, h, 1000 + k).view(torch.uint8).reshape(-1)
        else:
            f = workloads.field_frame_torch(w, h, 1000 + k).view(torch.uint8).reshape(-1)
        frames.append((f.contiguous(), w, h))
    files = [None] * n
    for ptype in (1, 2):
        for tile in SHAPES:
            group = [k for k in range(n) if types[k] == ptype and shapes[k] == tile]
            if group:
                s = 2 if ptype == 1 else 4
                encoded = encode_on_gpu(torch, stream, [(frames[k][0], frames[k][1], frames[k][2],
                                                         frames[k][1] * s) for k in group],
                                        ptype, tile)
                for k, f in zip(group, encoded):
                    files[k] = f
    entries, keep, decoded_bytes, alg = [], [], 0, 0
    plans = []
    for k in range(n):
        w, h = frames[k][1], frames[k][2]
        s = 2 if types[k] == 1 else 4
        st, meta = api.parse_metadata(files[k])
        assert st == Status.success
        src_dev = torch.from_numpy(np.frombuffer(files[k], dtype=np.uint8).copy()).cuda()
        pitch = (w * s + 127) // 128 * 128
        out = torch.empty(pitch * h, dtype=torch.uint8, device="cuda")
        src = CompressedInput()
        src.bytes = ConstBytes(src_dev.data_ptr(), len(files[k]))
        src.metadata = meta.handle
        item = BatchItem()
        item.compressed_input = src
        item.output = api.view(out, int(types[k]), w, h, pitch)
        entries.append((cuda.Operation.decompress, item))
        keep += [meta, src_dev, out]
        decoded_bytes += w * h * s
        t = meta.tiles
        alg += int(t["length"].sum()) + 32 * len(t) + w * h * s
        st, plan = cuda.prepare_batch(cuda.make_request(cuda.Operation.decompress, [item]),
                                      None, stream)
        assert st == Status.success
        plans.append((plan, out, pitch, w, h, s))
    return entries, plans, frames, keep, decoded_bytes, alg


def run_batched(args, torch, stream, peak):
    """Config 4: 256 archives with width and height uniform in 257..4096, 70% uint16 / 30%
    float32, a random tile geometry each, decoded into pitched rows: one mixed batch (one
    persistent kernel, CUDA graph, autotuned) against per-image plain decode on the same GPU."""
    from tilestream_b200 import cuda
    from tilestream_b200.api import Status
    n = args.archives
    entries, plans, frames, keep, decoded_bytes, alg = mixed_archives(torch, stream, n)
    results = torch.zeros(16 * n, dtype=torch.uint8, device="cuda")
    t0 = time.perf_counter()
    st, batch = cuda.prepare_mixed_batch(entries, results, stream, graph=True, autotune=True)
    prepare_s = time.perf_counter() - t0
    assert st == Status.success, st
    assert batch.run(stream) == Status.success
    torch.cuda.synchronize()
    exact = True
    for k, (plan, out, pitch, w, h, s) in enumerate(plans):
        rows = out.view(h, pitch)[:, :w * s]
        exact = exact and bool(torch.equal(rows, frames[k][0].view(h, w * s)))
    recs = results.cpu().numpy().view(np.uint64).reshape(-1, 2)
    exact = exact and bool(np.all(recs[:, 0] == 0))
    steps = max(3, args.steps // 300)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(args.warmup):
        batch.run(stream)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        batch.run(stream)
    e1.record(stream)
    torch.cuda.synchronize()
    batched_ms = e0.elapsed_time(e1) / steps

    # The device work queue against static striding: the same batch with fixed kernel shapes,
    # static (5, 6) and with the work queue (8, 9: the same shapes claiming task chunks).
    def fixed_ms(shape):
        st_f, b = cuda.prepare_mixed_batch(entries, results, stream, graph=True, shape=shape)
        assert st_f == Status.success, st_f
        for _ in range(args.warmup):
            b.run(stream)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            b.run(stream)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps
    queue = {}
    for static, dynamic in ((5, 8), (6, 9)):
        a, b = fixed_ms(static), fixed_ms(dynamic)
        queue[f"shape{static}_static_ms"] = round(a, 4)
        queue[f"shape{dynamic}_work_queue_ms"] = round(b, 4)

    ws = torch.empty(max(max(p[0].workspace_bytes() for p in plans), 256), dtype=torch.uint8,
                     device="cuda")
    res1 = torch.zeros(16, dtype=torch.uint8, device="cuda")

    def per_image():
        for plan, *_ in plans:
            cuda.decompress_async(plan, ws, res1, stream)

    per_image()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        per_image()
    e1.record(stream)
    torch.cuda.synchronize()
    eager_ms = e0.elapsed_time(e1) / steps
    graphed_ms = time_graph(torch, stream, per_image, steps, args.warmup)
    return {"workload": f"{n} archives, width/height uniform 257..4096, 70% uint16 / 30% "
                        "float32, random tile geometry, pitched output rows, whole-image decode",
            "decoded_bytes": decoded_bytes,
            "batched": {"ms": round(batched_ms, 4),
                        "decoded_gbs": round(decoded_bytes / batched_ms / 1e6, 1),
                        "roofline_frac": round(alg / batched_ms / 1e6 / peak, 4),
                        "hbm_gbs": round(alg / batched_ms / 1e6, 1),
                        "kernel_launches": 1, "prepare_s": round(prepare_s, 3),
                        **batch.stats()},
            "per_image_eager": {"ms": round(eager_ms, 4),
                                "decoded_gbs": round(decoded_bytes / eager_ms / 1e6, 1),
                                "kernel_launches": n},
            "per_image_graph": {"ms": round(graphed_ms, 4),
                                "decoded_gbs": round(decoded_bytes / graphed_ms / 1e6, 1)},
            "speedup_vs_per_image_eager": round(eager_ms / batched_ms, 2),
            "speedup_vs_per_image_graph": round(graphed_ms / batched_ms, 2),
            "work_queue_vs_static": queue,
            "bit_exact": exact}


def run_encode(args, torch, stream, peak, shapes):
    """Encoder on the headline frame: one compress plan per tile geometry, each step encodes the
    uint16 4096x4096 frame once, rotating over 4 input/output copies (more than the L2 holds),
    replayed as a CUDA graph. Bitstreams are checked against the archives the headline decodes
    (which the tests check byte for byte against the CPU codec)."""
    from tilestream_b200 import api, cuda, workloads
    from tilestream_b200.api import BatchItem, Status, TileShape
    frame = workloads.detector_frame(W, H, seed=SEED)
    copies = 4
    srcs = [torch.from_numpy(frame.view(np.uint8).reshape(-1).copy()).cuda()
            for _ in range(copies)]
    out = {}
    for s in shapes:
        tile = TileShape(*s["tile"])
        st, bound = api.compress_bound(api.image_spec(1, W, H), tile)
        runs = []
        for c in range(copies):
            dst = torch.empty(bound, dtype=torch.uint8, device="cuda")
            item = BatchItem()
            item.input = api.const_view(srcs[c], 1, W, H, W * 2)
            item.compressed_output = api.MutableBytes(dst.data_ptr(), bound)
            st, plan = cuda.prepare_batch(cuda.make_request(cuda.Operation.compress, [item],
                                                            tile), None, stream)
            assert st == Status.success, st
            ws = torch.empty(plan.workspace_bytes(), dtype=torch.uint8, device="cuda")
            res = torch.zeros(16, dtype=torch.uint8, device="cuda")
            runs.append((plan, ws, res, dst))

        def step():
            for plan, ws, res, _ in runs:
                cuda.compress_async(plan, ws, res, stream)

        step()
        torch.cuda.synchronize()
        for plan, ws, res, dst in runs:
            size = int(res.cpu().numpy().view(np.uint64)[1])
            assert int(res.cpu().numpy().view(np.uint32)[0]) == 0
            assert dst[:size].cpu().numpy().tobytes() == s["file"], "encoder bytes differ"
        ms = time_graph(torch, stream, step, max(3, args.steps // 200), args.warmup) / copies
        alg = W * H * 2 + len(s["file"])
        out["%dx%d" % s["tile"]] = {
            "launch_us": round(ms * 1e3, 2), "input_gbs": round(W * H * 2 / ms / 1e6, 1),
            "hbm_gbs": round(alg / ms / 1e6, 1), "roofline_frac": round(alg / ms / 1e6 / peak, 4),
            "bytes_equal": True}
    return {"workload": "uint16 4096x4096 frame (seed 2), one compress plan per tile geometry, "
                        "4 rotating copies, CUDA graph replay",
            "algorithmic_bytes": "input pixels + output file bytes", **out}


def serve_summary(stats, count):
    return {"requests": count, "completed": stats.completed,
            "p50_ms": round(stats.p50_us / 1e3, 4), "p90_ms": round(stats.p90_us / 1e3, 4),
            "p99_ms": round(stats.p99_us / 1e3, 4), "max_ms": round(stats.max_us / 1e3, 4),
            "mean_ms": round(stats.mean_us / 1e3, 4),
            "throughput_rps": round(stats.throughput_rps, 1),
            "decoded_gbs": round(stats.decoded_gbs, 2), "wall_s": round(stats.wall_us / 1e6, 4),
            "launches": stats.batches, "mean_batch": round(stats.mean_batch, 3),
            "max_inflight": stats.max_inflight, "stalls": stats.stalls, "tiles": stats.tiles}


class _DeviceBytes:
    """A view of device memory that the library owns (a server's output pool) for torch."""

    def __init__(self, address: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1",
                                         "data": (address, False), "version": 3}


def serving_calibration_error(torch, n, side, rate, resident, metas):
    """Served FP32 calibrated outputs against FP64 and against the host two-rounding form
    (x - offset, then times gain, each rounded to binary32): the calibrated requests among 200
    of the serving distribution (seed 8), outputs kept in the pool and read back."""
    from tilestream_b200 import cuda, workloads
    from tilestream_b200.api import ConstBytes, Status
    arrays = workloads.serving_requests(200, n, side, side, rate, seed=8)
    keep = np.flatnonzero(arrays["calibrated"])
    arrays = {k: v[keep] for k, v in arrays.items()}
    w, h = arrays["width"].astype(np.int64), arrays["height"].astype(np.int64)
    need = int((((w * 4 + 15) // 16 * 16 * h + 255) // 256 * 256).sum())
    srv = cuda.Server(pool_bytes=need, max_batch=48, max_inflight=4, retain_outputs=True)
    for dev, meta in zip(resident, metas):
        st, _ = srv.add_archive(ConstBytes(dev.data_ptr(), dev.numel()), meta, owner=dev)
        assert st == Status.success, st
    assert srv.seal() == Status.success
    st, outcomes, _ = srv.run(cuda.serve_requests(arrays))
    assert st == Status.success, st
    torch.cuda.synchronize()
    p = srv.pool()
    pool = torch.as_tensor(_DeviceBytes(p.data, need), device="cuda")
    worst, same, pixels, frame, current, contract = 0.0, True, 0, None, -1, None
    for i in np.argsort(arrays["archive"], kind="stable"):  # one source frame at a time
        oc = outcomes[int(i)]
        assert oc.result.status == 0, (i, oc.result.status)
        a = int(arrays["archive"][i])
        if a != current:
            frame, current = workloads.detector_frame_torch(side, side, 5000 + a), a
        x0, y0, rw, rh = (int(arrays[k][i]) for k in ("x", "y", "width", "height"))
        x = frame[y0:y0 + rh, x0:x0 + rw].cpu().numpy().astype(np.float32)
        rows = pool[oc.output_offset:oc.output_offset + oc.output_pitch * rh].view(rh, -1)
        got = rows[:, :rw * 4].contiguous().view(torch.float32).cpu().numpy()
        o, g = np.float32(arrays["offset"][i]), np.float32(arrays["gain"][i])
        host_form = ((x - o).astype(np.float32) * g).astype(np.float32)
        same = same and bool(np.array_equal(got.view(np.uint32), host_form.view(np.uint32)))
        ref = (x.astype(np.float64) - float(o)) * float(g)
        normal = np.abs(ref) >= 2.0 ** -126
        ulp = np.spacing(np.abs(ref[normal]).astype(np.float32)).astype(np.float64)
        if ulp.size:
            worst = max(worst, float(np.max(np.abs(got[normal] - ref[normal]) / ulp)))
        contract = merge_contract(contract, calibration_contract(x, o, g, got))
        pixels += rw * rh
    del pool, srv  # the view first: the pool's memory belongs to the server
    return {"requests": int(len(keep)), "pixels": int(pixels),
            "equals_host_two_rounding_form": same,
            "max_ulp_vs_fp64_normal_results": round(worst, 4), "ulp_bound": 1.5,
            "contract": contract}


def run_serving(args, torch, stream):
    """Config 5: 64 uint16 8192x8192 archives with 64x64 tiles resident in device memory; a
    request stream with Poisson arrivals at 20k req/s, each an ROI with sides log-uniform in
    32..4096 px at a uniform offset, 40% with fused scalar calibration (offset 100.0, gain 1.05).
    Continuous batching against one request at a time (resident tables, and the plan API)."""
    from tilestream_b200 import api, cuda, workloads
    from tilestream_b200.api import ConstBytes, Status
    n, side, tile = args.serve_archives, 8192, (64, 64)
    files = []
    for g in range(0, n, 8):
        frames = [workloads.detector_frame_torch(side, side, 5000 + k).view(torch.uint8)
                  .reshape(-1).contiguous() for k in range(g, min(n, g + 8))]
        files += encode_on_gpu(torch, stream, [(f, side, side, side * 2) for f in frames], 1,
                               tile)
        del frames
    resident, metas, compressed = [], [], 0
    for f in files:
        st, meta = api.parse_metadata(f)
        assert st == Status.success, st
        dev = torch.from_numpy(np.frombuffer(f, dtype=np.uint8).copy()).cuda()
        resident.append(dev)
        metas.append(meta)
        compressed += len(f)
    del files
    rate = args.serve_rate
    stream_arrays = workloads.serving_requests(args.serve_requests, n, side, side, rate, seed=5)
    requests = cuda.serve_requests(stream_arrays)
    serial_count = min(len(requests), args.serve_serial_requests)
    serial_requests = (cuda.N.ServeRequest * serial_count)(*requests[:serial_count])
    warm = workloads.serving_requests(200, n, side, side, rate, seed=6)
    results, servers = {}, {}
    for name, options, reqs in (
            ("continuous_batching", dict(max_batch=48, max_inflight=4), requests),
            ("one_at_a_time_resident", dict(max_batch=1, max_inflight=1), requests),
            ("one_at_a_time_plan", dict(serial=True), serial_requests)):
        srv = cuda.Server(pool_bytes=args.serve_pool_gb << 30, **options)
        for dev, meta in zip(resident, metas):
            st, _ = srv.add_archive(ConstBytes(dev.data_ptr(), dev.numel()), meta, owner=dev)
            assert st == Status.success, st
        assert srv.seal() == Status.success
        st, _, _ = srv.run(cuda.serve_requests(warm))
        assert st == Status.success, st
        st, outcomes, stats = srv.run(reqs)
        assert st == Status.success, st
        ok = all(outcomes[i].result.status == 0 for i in range(len(reqs)))
        results[name] = {**serve_summary(stats, len(reqs)), "all_success": ok}
        servers[name] = srv
    # Offered rate sweep (same request distribution, 10,000 requests per point): where
    # continuous batching and one request at a time part.
    sweep = []
    for r in args.serve_sweep:
        arrays = workloads.serving_requests(10000, n, side, side, r, seed=7)
        point = {"offered_rps": r}
        for name in ("continuous_batching", "one_at_a_time_resident"):
            st, outcomes, stats = servers[name].run(cuda.serve_requests(arrays))
            assert st == Status.success, st
            point[name] = {k: v for k, v in serve_summary(stats, 10000).items()
                           if k in ("p50_ms", "p99_ms", "throughput_rps", "decoded_gbs",
                                    "mean_batch", "max_inflight", "stalls")}
        sweep.append(point)
    results["rate_sweep"] = sweep
    servers.clear()
    results["calibration_error"] = serving_calibration_error(torch, n, side, rate, resident,
                                                             metas)
    area = stream_arrays["width"].astype(np.float64) * stream_arrays["height"]
    return {"workload": f"{n} uint16 {side}x{side} archives, 64x64 tiles, resident; Poisson "
                        f"arrivals at {rate:.0f} req/s; ROI sides log-uniform 32..4096 at a "
                        "uniform offset; 40% fused scalar calibration (offset 100.0, gain 1.05)",
            "resident_compressed_gb": round(compressed / 1e9, 3),
            "mean_roi_mpx": round(float(area.mean()) / 1e6, 4),
            "calibrated_fraction": round(float(stream_arrays["calibrated"].mean()), 4),
            "offered_gbs": round(float((area * np.where(stream_arrays["calibrated"], 4, 2))
                                       .sum()) / (float(stream_arrays["arrival_us"][-1]) * 1e3),
                                 2),
            **results,
            "p99_under_1ms": results["continuous_batching"]["p99_ms"] < 1.0,
            "latency": "arrival (host clock, Poisson schedule) to completion seen by the "
                       "serving loop polling the launch's event"}


def run_profile_case(kind: str, launches: int = 3):
    """A small case for ncu captures: one launch of `kind` over four 4096x4096 frames (about
    216 MB of decode traffic, more than the 126 MB L2), repeated `launches` times; `step` is
    the headline step itself (the three archives in one launch, about 162 MB); `field`,
    `calibrate`, `batch` and `serve` are one launch of the fused FP32 decode, the standalone
    calibration, the mixed batch and the serving kernel on smaller copies of their configs;
    `stage` stages one ROI's payloads from pinned host memory."""
    import torch
    from tilestream_b200 import api, cuda, workloads
    from tilestream_b200.api import BatchItem, CompressedInput, ConstBytes, Status, TileShape
    stream = torch.cuda.current_stream()
    if kind == "calibrate":
        # The standalone calibration kernel: a float32 4096x4096 frame with FP32 offset and gain
        # maps (16 B per pixel, 268 MB per launch).
        field = workloads.field_frame(W, H, seed=3)
        offset, gain = workloads.calibration_maps(W, H, seed=5)
        frame_dev, off_dev, gain_dev = [torch.from_numpy(a.view(np.uint8).reshape(-1).copy())
                                        .cuda() for a in (field, offset, gain)]
        out = torch.empty(W * H * 4, dtype=torch.uint8, device="cuda")
        item = BatchItem()
        item.input = api.const_view(frame_dev, 2, W, H, W * 4)
        item.output = api.view(out, 2, W, H, W * 4)
        item.calibration.offset.kind = cuda.ParameterKind.map
        item.calibration.offset.map = api.const_view(off_dev, 2, W, H, W * 4)
        item.calibration.gain.kind = cuda.ParameterKind.map
        item.calibration.gain.map = api.const_view(gain_dev, 2, W, H, W * 4)
        st, plan = cuda.prepare_batch(cuda.make_request(cuda.Operation.calibrate, [item]), None,
                                      stream)
        assert st == Status.success, st
        res = torch.zeros(16, dtype=torch.uint8, device="cuda")
        for _ in range(launches):
            assert cuda.calibrate_async(plan, None, res, stream) == Status.success
        torch.cuda.synchronize()
        assert int(res.cpu().numpy().view(np.uint32)[0]) == 0
        print(json.dumps({"profile_case": kind, "launches": launches, "images_per_launch": 1}))
        return
    if kind == "batch":
        # Config 4's mixed batch on 48 of its archives (about 0.6 GB decoded), graph replay.
        # The autotuner's choice is kept in the file TILESTREAM_TUNE_CACHE names, so a second
        # run of the same command (the one under ncu) launches no trial kernels.
        n = 48
        entries, plans, frames, keep, decoded, alg = mixed_archives(torch, stream, n)
        results = torch.zeros(16 * n, dtype=torch.uint8, device="cuda")
        st, batch = cuda.prepare_mixed_batch(entries, results, stream, graph=True,
                                             autotune=True)
        assert st == Status.success, st
        for _ in range(launches):
            assert batch.run(stream) == Status.success
        torch.cuda.synchronize()
        assert np.all(results.cpu().numpy().view(np.uint64).reshape(-1, 2)[:, 0] == 0)
        print(json.dumps({"profile_case": kind, "launches": launches, "images_per_launch": n,
                          "decoded_bytes": decoded, "algorithmic_bytes": alg,
                          **batch.stats()}))
        return
    if kind == "serve":
        # Config 5's serving kernel: 4 uint16 8192x8192 archives with 64x64 tiles resident and
        # 48 x launches requests of its ROI distribution that all arrive at once, so each launch
        # serves 48 requests.
        from tilestream_b200.api import ConstBytes
        side, count = 8192, 4
        frames = [workloads.detector_frame_torch(side, side, 5000 + k).view(torch.uint8)
                  .reshape(-1).contiguous() for k in range(count)]
        files = encode_on_gpu(torch, stream, [(f, side, side, side * 2) for f in frames], 1,
                              (64, 64))
        del frames
        srv = cuda.Server(pool_bytes=1 << 30, max_batch=48, max_inflight=1)
        for f in files:
            st, meta = api.parse_metadata(f)
            assert st == Status.success, st
            dev = torch.from_numpy(np.frombuffer(f, dtype=np.uint8).copy()).cuda()
            st, _ = srv.add_archive(ConstBytes(dev.data_ptr(), dev.numel()), meta, owner=dev)
            assert st == Status.success, st
        assert srv.seal() == Status.success
        arrays = workloads.serving_requests(48 * launches, count, side, side, 1e12, seed=5)
        st, outcomes, stats = srv.run(cuda.serve_requests(arrays))
        assert st == Status.success, st
        assert all(outcomes[i].result.status == 0 for i in range(48 * launches))
        area = arrays["width"].astype(np.int64) * arrays["height"]
        print(json.dumps({"profile_case": kind, "launches": stats.batches,
                          "requests": 48 * launches, "mean_batch": round(stats.mean_batch, 2),
                          "decoded_bytes": int((area * np.where(arrays["calibrated"], 4, 2))
                                               .sum())}))
        return
    if kind == "stage":
        # The ROI staging kernel: the payloads of a 2048x2048 ROI (64 tile rows of 16 tiles, one
        # run each) of the seed-2 frame's 128x32 archive, read from pinned host memory.
        from tilestream_b200.api import MutableBytes, Roi, TileMapping
        frame = workloads.detector_frame(W, H, seed=SEED)
        dev_frame = torch.from_numpy(frame.view(np.uint8).reshape(-1).copy()).cuda()
        file = encode_on_gpu(torch, stream, [(dev_frame, W, H, W * 2)], 1, (128, 32))[0]
        del dev_frame
        st, meta = api.parse_metadata(file)
        assert st == Status.success, st
        pinned = torch.from_numpy(np.frombuffer(file, dtype=np.uint8).copy()).pin_memory()
        roi = Roi(1024, 1024, 2048, 2048)
        st, need = cuda.roi_staging_size(meta, roi)
        assert st == Status.success, st
        staging = torch.empty(need.bytes, dtype=torch.uint8, device="cuda")
        maps = (TileMapping * need.tiles)()
        for _ in range(launches):
            st, got = cuda.stage_roi_tiles(meta, roi, ConstBytes(pinned.data_ptr(), len(file)),
                                           MutableBytes(staging.data_ptr(), need.bytes), maps,
                                           stream)
            assert st == Status.success, st
        torch.cuda.synchronize()
        host = staging.cpu().numpy()
        tiles = meta.tiles
        for m in maps:
            t = int(m.tile_index)
            a, n = int(tiles["offset"][t]), int(tiles["length"][t])
            assert host[m.input_offset:m.input_offset + n].tobytes() == file[a:a + n]
        print(json.dumps({"profile_case": kind, "launches": launches, "tiles": need.tiles,
                          "bytes": need.bytes, "copies": need.copies}))
        return
    if kind == "field":
        # Config 3's fused launch: the float32 field decoded with FP32 offset and gain maps.
        field = workloads.field_frame(W, H, seed=3)
        offset, gain = workloads.calibration_maps(W, H, seed=5)
        dev_frame = torch.from_numpy(field.view(np.uint8).reshape(-1).copy()).cuda()
        file = encode_on_gpu(torch, stream, [(dev_frame, W, H, W * 4)], 2, (128, 32))[0]
        st, meta = api.parse_metadata(file)
        src_dev = torch.from_numpy(np.frombuffer(file, dtype=np.uint8).copy()).cuda()
        maps = [torch.from_numpy(m.view(np.uint8).reshape(-1).copy()).cuda()
                for m in (offset, gain)]
        out = torch.empty(W * H * 4, dtype=torch.uint8, device="cuda")
        src = CompressedInput()
        src.bytes = ConstBytes(src_dev.data_ptr(), len(file))
        src.metadata = meta.handle
        item = BatchItem()
        item.compressed_input = src
        item.output = api.view(out, 2, W, H, W * 4)
        item.roi = api.Roi(0, 0, W, H)
        item.calibration.offset.kind = cuda.ParameterKind.map
        item.calibration.offset.map = api.const_view(maps[0], 2, W, H, W * 4)
        item.calibration.gain.kind = cuda.ParameterKind.map
        item.calibration.gain.map = api.const_view(maps[1], 2, W, H, W * 4)
        st, plan = cuda.prepare_batch(cuda.make_request(cuda.Operation.decode_calibrate, [item]),
                                      None, stream)
        assert st == Status.success, st
        ws = torch.empty(max(plan.workspace_bytes(), 256), dtype=torch.uint8, device="cuda")
        res = torch.zeros(16, dtype=torch.uint8, device="cuda")
        for _ in range(launches):
            assert cuda.decode_calibrate_async(plan, ws, res, stream) == Status.success
        torch.cuda.synchronize()
        assert int(res.cpu().numpy().view(np.uint32)[0]) == 0
        print(json.dumps({"profile_case": kind, "launches": launches, "images_per_launch": 1}))
        return
    if kind == "unparsed":
        # The headline step's three archives decoded as unparsed files (decode_unparsed_async:
        # index entries, payloads and rows validated on the device), one launch each time.
        frame, shapes, step_plans, workspace, results = prepare_workload(torch, stream, 1)
        entries = [(ConstBytes(s["copies"][0]["src"].data_ptr(), len(s["file"])), s["file"][:64],
                    api.view(s["copies"][0]["out"], 1, W, H, W * 2)) for s in shapes]
        for _ in range(launches):
            assert cuda.decode_unparsed_async(entries, api.ResultBuffer(results.data_ptr(), 3),
                                              stream) == Status.success
        torch.cuda.synchronize()
        recs = results.cpu().numpy().view(np.uint64).reshape(-1, 2)[:3]
        assert all(int(r[0]) == 0 for r in recs), recs
        for s in shapes:
            assert np.array_equal(s["copies"][0]["out"].cpu().numpy().view(np.uint16),
                                  frame.reshape(-1))
        print(json.dumps({"profile_case": kind, "launches": launches, "images_per_launch": 3}))
        return
    if kind == "step":
        frame, shapes, step_plans, workspace, results = prepare_workload(torch, stream, 1)
        wsb = api.MutableBytes(workspace.data_ptr(), workspace.numel())
        for _ in range(launches):
            assert cuda.decompress_async(step_plans[0], wsb, api.ResultBuffer(
                results.data_ptr(), 3), stream) == Status.success
        torch.cuda.synchronize()
        for s in shapes:
            assert np.array_equal(s["copies"][0]["out"].cpu().numpy().view(np.uint16),
                                  frame.reshape(-1))
        print(json.dumps({"profile_case": kind, "launches": launches, "images_per_launch": 3}))
        return
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
        dev_frame = torch.from_numpy(frame.view(np.uint8).reshape(-1).copy()).cuda()
        file = encode_on_gpu(torch, stream, [(dev_frame, W, H, W * 2)], 1, (128, 32))[0]
        del dev_frame
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
    p.add_argument("--profile", choices=["decode", "fused", "encode", "step", "field",
                                         "calibrate", "batch", "serve", "stage", "unparsed"],
                   default=None,
                   help="run only a small case for ncu captures and exit")
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3000)
    p.add_argument("--warmup", type=int, default=20)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--copies", type=int, default=4)
    p.add_argument("--min-span-ms", type=float, default=200.0,
                   help="the K-step timed region repeats until the repetitions span this long")
    p.add_argument("--max-regions", type=int, default=5000)
    p.add_argument("--cpu-seconds", type=float, default=10.0)
    p.add_argument("--sections", default="encode,calibrated,batched,serving,archive_roi",
                   help="extra configs reported beside the headline (comma list, or none)")
    p.add_argument("--archives", type=int, default=256, help="archives of the batched config")
    p.add_argument("--serve-archives", type=int, default=64)
    p.add_argument("--serve-requests", type=int, default=20000)
    p.add_argument("--serve-serial-requests", type=int, default=2000,
                   help="requests of the one-at-a-time plan-API baseline")
    p.add_argument("--serve-rate", type=float, default=20000.0, help="offered requests/s")
    p.add_argument("--serve-pool-gb", type=int, default=2)
    p.add_argument("--serve-sweep", type=lambda v: [float(x) for x in v.split(",") if x],
                   default=[50000.0, 100000.0, 200000.0, 400000.0],
                   help="offered rates (req/s) of the serving sweep")
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
        # The configs' sections, the host parse and the CPU baseline run at N = 1 only: a
        # scaling run measures the headline step, and the other ranks would wait in the final
        # barrier (whose timeout is short) while rank 0 ran them.
        sections = [s for s in args.sections.split(",") if s and s != "none"] if world == 1 \
            else []
        stream = torch.cuda.current_stream()
        peak = measured_peaks()[0]
        if "encode" in sections:
            line["encode"] = run_encode(args, torch, stream, peak, shapes)
        if "calibrated" in sections:
            line["calibrated_decode"] = run_calibrated(args, torch, stream, peak)
        if "batched" in sections:
            line["batched_decode"] = run_batched(args, torch, stream, peak)
        if "serving" in sections:
            line["serving"] = run_serving(args, torch, stream)
        if "archive_roi" in sections:
            line["archive_roi"] = run_archive_roi(args, torch, shapes)
        if world == 1:
            line["host_parse"] = host_parse(shapes)
            line["cpu_baseline"] = cpu_baseline(shapes, args.cpu_seconds)
        else:
            line["cpu_baseline"] = None  # measured at N = 1
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
