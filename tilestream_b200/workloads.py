"""Seeded synthetic frames with the shapes and value distributions of the benchmark configs.

The reference quotes its numbers on synthetic detector frames; these generators stand in for
them with fixed RNGs so that every run (here, in tests and on the GPU host) sees the same
pixels:

* `detector_frame`  uint16: clamp(round(1000 + 200 sin(x/97) cos(y/61) + N(0, 12)), 0, 65535),
  0.5 % hot pixels at 65535 and 1 % of the 128x32 tile grid set constant (configs 1, 2, 4, 5).
* `field_frame`     float32 words: 500 + 50 sin(x/211) + 30 cos(y/173) + N(0, 0.5), low 8
  mantissa bits random, 0.1 % special words (+-0, +-inf, NaN with random payloads, subnormals)
  (configs 3 and 4).
* `calibration_maps` offset ~ N(100, 5), gain ~ U(0.9, 1.1) FP32 maps (config 3).
* `serving_requests` a request stream: Poisson arrivals, ROI sides log-uniform in [32, 4096]
  at a uniform offset inside the archive, 40 % with scalar calibration (offset 100.0, gain
  1.05) (config 5).

RNG: numpy PCG64 seeded with the frame seed; sin/cos come from the C library through `math` on
1-D axes, so results do not depend on numpy's SIMD transcendental kernels. The `*_torch`
variants generate the same distributions on the GPU (torch's Philox generator, seeded) for the
multi-gigabyte batched and serving workloads, where host generation would dominate the run.
"""
from __future__ import annotations

import math

import numpy as np

HOT_FRACTION = 0.005
CONSTANT_TILE_FRACTION = 0.01
SPECIAL_FRACTION = 0.001


def _axis(n: int, fn, scale: float) -> np.ndarray:
    return np.array([fn(i / scale) for i in range(n)], dtype=np.float64)


def detector_frame(width: int, height: int, seed: int) -> np.ndarray:
    """uint16 detector frame, shape (height, width)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sx = _axis(width, math.sin, 97.0)
    cy = _axis(height, math.cos, 61.0)
    noise = rng.normal(0.0, 12.0, size=(height, width))
    values = 1000.0 + 200.0 * (cy[:, None] * sx[None, :]) + noise
    frame = np.clip(np.rint(values), 0, 65535).astype(np.uint16)
    hot = rng.random((height, width)) < HOT_FRACTION
    frame[hot] = 65535
    _constant_tiles(frame, rng)
    return frame


def _constant_tiles(frame: np.ndarray, rng: np.random.Generator) -> None:
    """Sets 1 % of the 128x32 tile grid (at least one tile) to its first pixel's value."""
    height, width = frame.shape
    across = -(-width // 128)
    down = -(-height // 32)
    count = max(1, int(round(CONSTANT_TILE_FRACTION * across * down)))
    for t in rng.choice(across * down, size=count, replace=False):
        x, y = int(t % across) * 128, int(t // across) * 32
        frame[y:y + 32, x:x + 128] = frame[y, x]


def field_frame(width: int, height: int, seed: int) -> np.ndarray:
    """float32 smooth field as uint32 bit words, shape (height, width)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sx = _axis(width, math.sin, 211.0)
    cy = _axis(height, math.cos, 173.0)
    values = 500.0 + 50.0 * sx[None, :] + 30.0 * cy[:, None] + rng.normal(0.0, 0.5,
                                                                         (height, width))
    words = values.astype(np.float32).view(np.uint32)
    words = (words & np.uint32(0xFFFFFF00)) | rng.integers(0, 256, (height, width),
                                                           dtype=np.uint32)
    special = rng.random((height, width)) < SPECIAL_FRACTION
    n = int(special.sum())
    kind = rng.integers(0, 6, n)
    sign = rng.integers(0, 2, n, dtype=np.uint32) << np.uint32(31)
    mantissa = rng.integers(1, 1 << 23, n, dtype=np.uint32)
    table = np.select(
        [kind == 0, kind == 1, kind == 2, kind == 3, kind == 4],
        [np.uint32(0), np.uint32(0x80000000), np.uint32(0x7F800000), np.uint32(0xFF800000),
         sign | np.uint32(0x7F800000) | mantissa],
        default=sign | mantissa)  # subnormal: exponent 0, nonzero mantissa
    words[special] = table.astype(np.uint32)
    return words


def calibration_maps(width: int, height: int, seed: int):
    """FP32 offset ~ N(100, 5) and gain ~ U(0.9, 1.1) maps, shape (height, width)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    offset = rng.normal(100.0, 5.0, (height, width)).astype(np.float32)
    gain = rng.uniform(0.9, 1.1, (height, width)).astype(np.float32)
    return offset, gain


# --- GPU-side generators for the large batched and serving workloads -------------------------

def detector_frame_torch(width: int, height: int, seed: int, device="cuda"):
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    x = torch.arange(width, device=device, dtype=torch.float64)
    y = torch.arange(height, device=device, dtype=torch.float64)
    base = 1000.0 + 200.0 * torch.cos(y / 61.0)[:, None] * torch.sin(x / 97.0)[None, :]
    noise = torch.randn((height, width), generator=g, device=device, dtype=torch.float32) * 12.0
    frame = torch.clamp(torch.round(base + noise), 0, 65535).to(torch.int32)
    hot = torch.rand((height, width), generator=g, device=device) < HOT_FRACTION
    frame[hot] = 65535
    across, down = -(-width // 128), -(-height // 32)
    count = max(1, int(round(CONSTANT_TILE_FRACTION * across * down)))
    picks = torch.randperm(across * down, generator=g, device=device)[:count].tolist()
    for t in picks:
        tx, ty = (t % across) * 128, (t // across) * 32
        frame[ty:ty + 32, tx:tx + 128] = frame[ty, tx].item()
    return frame.to(torch.uint16)


def field_frame_torch(width: int, height: int, seed: int, device="cuda"):
    """float32 field as int32 words (bit patterns), shape (height, width)."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    x = torch.arange(width, device=device, dtype=torch.float64)
    y = torch.arange(height, device=device, dtype=torch.float64)
    values = (500.0 + 50.0 * torch.sin(x / 211.0)[None, :] + 30.0 * torch.cos(y / 173.0)[:, None]
              + 0.5 * torch.randn((height, width), generator=g, device=device,
                                  dtype=torch.float64))
    words = values.to(torch.float32).view(torch.int32)
    low = torch.randint(0, 256, (height, width), generator=g, device=device, dtype=torch.int32)
    words = (words & ~0xFF) | low
    special = torch.rand((height, width), generator=g, device=device) < SPECIAL_FRACTION
    n = int(special.sum().item())
    if n:
        kind = torch.randint(0, 6, (n,), generator=g, device=device)
        sign = torch.randint(0, 2, (n,), generator=g, device=device, dtype=torch.int32) << 31
        mant = torch.randint(1, 1 << 23, (n,), generator=g, device=device, dtype=torch.int32)
        table = torch.where(kind == 0, torch.zeros_like(mant), sign | mant)
        table = torch.where(kind == 1, torch.full_like(mant, -0x80000000), table)
        table = torch.where(kind == 2, torch.full_like(mant, 0x7F800000), table)
        table = torch.where(kind == 3, torch.full_like(mant, -0x00800000), table)
        table = torch.where(kind == 4, sign | 0x7F800000 | mant, table)
        words[special] = table
    return words


def serving_requests(count: int, archives: int, width: int, height: int, rate_per_s: float,
                     seed: int, min_side: int = 32, max_side: int = 4096,
                     calibrated_fraction: float = 0.4, offset: float = 100.0,
                     gain: float = 1.05) -> dict:
    """A seeded request stream over `archives` archives of width x height pixels.

    Arrivals are a Poisson process of the given rate (exponential gaps, first request at the
    first gap). Each side is exp(U(ln min_side, ln max_side)) rounded, capped at the archive's
    size; the offset is uniform over the positions that keep the ROI inside the archive.
    Returns numpy arrays: arrival_us, archive, x, y, width, height, calibrated, offset, gain."""
    rng = np.random.Generator(np.random.PCG64(seed))
    gaps = rng.exponential(1e6 / rate_per_s, count)
    arrival = np.cumsum(gaps)
    lo = math.log(min_side)

    def sides(limit):
        hi = math.log(max(min(max_side, limit), min_side))
        v = np.rint(np.exp(rng.uniform(lo, hi, count))).astype(np.int64)
        return np.clip(v, min(min_side, limit), min(max_side, limit))

    w = sides(width)
    h = sides(height)
    x = (rng.random(count) * (width - w + 1)).astype(np.int64)
    y = (rng.random(count) * (height - h + 1)).astype(np.int64)
    archive = rng.integers(0, archives, count)
    calibrated = rng.random(count) < calibrated_fraction
    return {"arrival_us": arrival, "archive": archive, "x": x, "y": y, "width": w, "height": h,
            "calibrated": calibrated, "offset": np.full(count, offset, np.float32),
            "gain": np.full(count, gain, np.float32)}
