"""GPU parity at the configs' scale and on the reference's own inputs, all against the oracle:

* every accepted file of the reference's fuzz corpora (fuzz/corpus/parse, and the mutation
  corpus rebuilt into its files) decoded on the GPU equals the CPU decode;
* the reference's image fixtures (datasets/fixtures/*.npy) encode on the GPU to the oracle's
  bytes for every tile shape and decode back to the same words;
* a 4096x4096 FP32 field (config 3's generator) encodes byte-identically and decodes bit-exact;
* a config-4-sized mixed batch (sides 257..4096, uint16 and FP32, every tile shape, pitched
  input and output rows, calibration maps): every GPU-encoded file equals the oracle's, and every
  output of one mixed batch equals the oracle's words (calibrated outputs its two-rounding form);
* all 256 archives of the benchmark's config-4 batch encode to the oracle's bytes.
"""
import numpy as np
import pytest

import oracle
from support import SENTINEL, Run, device_bytes, gpu_decode, host, logical, to_device
from tilestream_b200 import api, cuda, workloads
from tilestream_b200.api import BatchItem, Status, TileShape

pytestmark = pytest.mark.gpu


def _gpu_matches_cpu(o, file):
    """Parses file; when accepted, its GPU decode equals the oracle's CPU decode (True), else
    False (rejected). Large images are skipped (None)."""
    st, meta = api.parse_metadata(np.frombuffer(file, np.uint8), size=len(file))
    if st != Status.success:
        return False
    image = meta.image
    if image.width * image.height > 1 << 22:
        return None
    want_st, want = o.decompress(file, image.type, image.width, image.height)
    assert want_st == 0
    gst, rec, out, pitch = gpu_decode(file)
    assert gst == Status.success and rec[0] == 0, rec
    s = api.sample_bytes(image.type)
    assert np.array_equal(logical(out, image.width, image.height, pitch, s),
                          np.frombuffer(want, np.uint8)[:image.width * image.height * s])
    return True


def test_fuzz_corpora_decode_on_gpu(cuda_ready, oracle_lib):
    from golden import inputs
    decoded = 0
    for name, data in inputs.corpus("parse"):
        decoded += bool(_gpu_matches_cpu(oracle_lib, data))
    for name, data in inputs.corpus("mutation"):
        file = oracle_lib.mutation_file(data)
        if file is not None:
            decoded += bool(_gpu_matches_cpu(oracle_lib, file))
    assert decoded > 100, decoded


def _encode_decode(o, words, ptype, tile, pitch=None):
    """GPU encode of (h, w) words (rows at `pitch` bytes) compared with the oracle's file, then
    GPU decode of that file compared with the words."""
    from test_gpu_encode import gpu_encode_many
    h, w = words.shape
    s = words.itemsize
    pitch = pitch or w * s
    buf = np.full(pitch * h, SENTINEL, np.uint8)
    for y in range(h):
        buf[y * pitch:y * pitch + w * s] = words[y].view(np.uint8)
    files, _ = gpu_encode_many([(buf, ptype, w, h, pitch)], tile=tile)
    want = o.compress_image(words, tile)
    assert files[0] == want, (w, h, tile)
    st, rec, out, opitch = gpu_decode(want)
    assert st == Status.success and rec[0] == 0
    assert np.array_equal(logical(out, w, h, opitch, s), words.view(np.uint8).reshape(-1))


def test_dataset_fixtures_on_gpu(cuda_ready, oracle_lib):
    from golden import inputs
    seen = 0
    for name, img in inputs.datasets():
        words = np.ascontiguousarray(img if img.dtype == np.uint16 else img.view(np.uint32))
        ptype = 1 if words.dtype == np.uint16 else 2
        for tile in api.TILE_SHAPES:
            _encode_decode(oracle_lib, words, ptype, tile)
        seen += 1
    assert seen == 4


def test_fp32_field_4096_encode_decode(cuda_ready, oracle_lib):
    """Config 3's FP32 4096x4096 field (0.1% special words), tiles 128x32, pitched input."""
    field = workloads.field_frame(4096, 4096, seed=3)
    _encode_decode(oracle_lib, field, 2, (128, 32), pitch=4096 * 4 + 64)


def _run_mixed(torch, stream, o, rng, words, types, files):
    from support import parsed_source
    items, keep, checks = [], [], []
    for k, file in enumerate(files):
        img = words[k]
        h, w = img.shape
        s = img.itemsize
        src, meta, dev = parsed_source(file)
        keep += [meta, dev]
        kind = k % 3
        if kind == 0:
            roi = (0, 0, w, h)
        else:
            x, y = int(rng.integers(0, w)), int(rng.integers(0, h))
            roi = (x, y, int(rng.integers(1, w - x + 1)), int(rng.integers(1, h - y + 1)))
        x, y, rw, rh = roi
        region = np.ascontiguousarray(img[y:y + rh, x:x + rw])
        item = BatchItem()
        item.compressed_input = src
        osz = 4 if kind == 2 else s
        pitch = (rw * osz + 127) // 128 * 128 + (16 if k % 2 else 0)
        out = device_bytes(pitch * rh)
        item.output = api.view(out, 2 if kind == 2 else int(types[k]), rw, rh, pitch, out.numel())
        op = cuda.Operation.decompress
        want = region.view(np.uint8).reshape(rh, rw * s)
        if kind >= 1:
            item.roi = api.Roi(*roi)
            op = cuda.Operation.decode_roi
        if kind == 2:
            op = cuda.Operation.decode_calibrate
            off, gain = workloads.calibration_maps(rw, rh, seed=500 + k)
            maps = [to_device(off), to_device(gain)]
            keep += maps
            item.calibration.offset.kind = cuda.ParameterKind.map
            item.calibration.offset.map = api.const_view(maps[0], 2, rw, rh, rw * 4)
            item.calibration.gain.kind = cuda.ParameterKind.map
            item.calibration.gain.map = api.const_view(maps[1], 2, rw, rh, rw * 4)
            want = o.calibrate_image(region, off, gain).view(np.uint8).reshape(rh, rw * 4)
        keep.append(out)
        items.append((op, item))
        checks.append((out, pitch, rw * osz, rh, want, kind == 2))
    results = device_bytes(16 * len(items), fill=0xFF)
    st, batch = cuda.prepare_mixed_batch(items, results, stream)
    assert st == Status.success, st
    assert batch.run(stream) == Status.success
    torch.cuda.synchronize()
    raw = host(results).view(np.uint64).reshape(-1, 2)
    for k, (out, pitch, row_bytes, rh, want, cal) in enumerate(checks):
        assert int(raw[k, 0]) == 0 and int(raw[k, 1]) == row_bytes * rh, k
        got = host(out)[:pitch * rh].reshape(rh, pitch)
        rows = np.ascontiguousarray(got[:, :row_bytes])
        if cal:
            a, b = rows.view(np.float32), np.ascontiguousarray(want).view(np.float32)
            assert np.all((a.view(np.uint32) == b.view(np.uint32)) |
                          (np.isnan(a) & np.isnan(b))), k
        else:
            assert np.array_equal(rows, want), k
        assert np.all(got[:, row_bytes:] == SENTINEL), k


def test_config4_sized_mixed_batch(cuda_ready, oracle_lib):
    """24 archives, sides uniform in 257..4096, 70% uint16 / 30% FP32, a random tile shape each,
    pitched input rows: GPU files equal the oracle's. Then one mixed batch over them - whole
    images, ROIs and ROIs calibrated with FP32 offset and gain maps, into pitched output rows -
    equals the oracle's words."""
    from test_gpu_encode import gpu_encode_many
    torch = cuda_ready
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(2024)
    n = 24
    dims = rng.integers(257, 4097, size=(n, 2))
    types = np.where(rng.random(n) < 0.7, 1, 2)
    tiles = [api.TILE_SHAPES[i] for i in rng.integers(0, 3, n)]
    words, files = [], [None] * n
    for k in range(n):
        w, h = int(dims[k, 0]), int(dims[k, 1])
        words.append(workloads.detector_frame(w, h, seed=100 + k) if types[k] == 1
                     else workloads.field_frame(w, h, seed=100 + k))
    for ptype in (1, 2):
        for tile in api.TILE_SHAPES:
            group = [k for k in range(n) if types[k] == ptype and tiles[k] == tile]
            if not group:
                continue
            images = []
            for k in group:
                img = words[k]
                h, w = img.shape
                pitch = w * img.itemsize + 4 * (1 + k % 5)
                buf = np.full(pitch * h, SENTINEL, np.uint8)
                buf.reshape(h, pitch)[:, :w * img.itemsize] = img.view(np.uint8).reshape(h, -1)
                images.append((buf, ptype, w, h, pitch))
            got, _ = gpu_encode_many(images, tile=tile)
            for k, f in zip(group, got):
                assert f == oracle_lib.compress_image(words[k], tile), (k, tile)
                files[k] = f
    _run_mixed(torch, stream, oracle_lib, rng, words, types, files)


def test_config4_every_archive_encodes_to_oracle_bytes(cuda_ready, oracle_lib):
    """All 256 archives of the benchmark's config-4 batch (bench.mixed_archives: sides uniform in
    257..4096, 70% uint16 / 30% FP32, a random tile shape each, generated and encoded on the
    GPU): every file equals the oracle's encoding of the same pixels, byte for byte."""
    import concurrent.futures as cf

    import bench
    torch = cuda_ready
    stream = torch.cuda.current_stream()
    entries, plans, frames, keep, _, _ = bench.mixed_archives(torch, stream, 256)
    torch.cuda.synchronize()

    def check(k):
        meta, src_dev = keep[3 * k], keep[3 * k + 1]
        dev, w, h = frames[k]
        pixels = dev.cpu().numpy()
        img = pixels.view(np.uint16 if meta.image.type == 1 else np.uint32)
        img = img.reshape(h, w) if meta.image.type == 1 else img.view(np.float32).reshape(h, w)
        want = oracle_lib.compress_image(np.ascontiguousarray(img),
                                         (meta.tile.width, meta.tile.height))
        return src_dev.cpu().numpy().tobytes() == want

    with cf.ThreadPoolExecutor(max_workers=8) as pool:
        same = list(pool.map(check, range(256)))
    assert all(same), [k for k, ok in enumerate(same) if not ok][:8]
