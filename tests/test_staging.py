"""ROI staging from an archive outside the GPU (include/tilestream/staging.h): sizes and the
checks that run before any copy, on the CPU. The copies and the decode of the staged tiles are
in test_gpu_staging.py."""
import numpy as np

from tilestream_b200 import api, cuda, workloads
from tilestream_b200.api import ConstBytes, MutableBytes, Roi, Status, TileMapping


def expected(meta, roi, tile):
    """Tiles, bytes and copies from the parsed tables: the ROI's tiles in row-major order, one
    copy per run of payloads that follow one another."""
    tiles = meta.tiles
    across = -(-meta.image.width // tile[0])
    x, y, w, h = roi
    count = nbytes = copies = 0
    begin = end = None
    for r in range(y // tile[1], (y + h - 1) // tile[1] + 1):
        for c in range(x // tile[0], (x + w - 1) // tile[0] + 1):
            t = r * across + c
            a = int(tiles["offset"][t])
            b = a + int(tiles["length"][t])
            if end is None or a != end:
                if end is not None:
                    nbytes += end - begin
                copies += 1
                begin = a
            end = b
            count += 1
    nbytes += end - begin
    return count, nbytes, copies


def test_sizes_match_tables(oracle_lib):
    rng = np.random.default_rng(7)
    frame = workloads.detector_frame(1000, 700, seed=3)
    for tile in api.TILE_SHAPES:
        file = oracle_lib.compress_image(frame, tile)
        st, meta = api.parse_metadata(np.frombuffer(file, dtype=np.uint8))
        assert st == Status.success
        rois = [(0, 0, 1000, 700), (999, 699, 1, 1), (0, 0, 1, 1), (tile[0] - 1, 0, 2, 700)]
        for _ in range(40):
            x, y = int(rng.integers(0, 1000)), int(rng.integers(0, 700))
            rois.append((x, y, int(rng.integers(1, 1001 - x)), int(rng.integers(1, 701 - y))))
        for roi in rois:
            st, r = cuda.roi_staging_size(meta, Roi(*roi))
            assert st == Status.success
            count, nbytes, copies = expected(meta, roi, tile)
            assert (r.tiles, r.bytes, r.copies) == (count, nbytes, copies)
            # A parsed file stores each tile row's payloads one after another: at most one
            # copy per tile row of the ROI (an ROI as wide as the image is one run).
            assert copies <= (roi[1] + roi[3] - 1) // tile[1] - roi[1] // tile[1] + 1


def test_checks_before_any_copy(oracle_lib):
    frame = workloads.detector_frame(300, 200, seed=6)
    file = oracle_lib.compress_image(frame)
    src = np.frombuffer(file, dtype=np.uint8)
    st, meta = api.parse_metadata(src)
    roi = Roi(10, 10, 200, 100)
    st, need = cuda.roi_staging_size(meta, roi)
    assert st == Status.success
    archive = ConstBytes(src.ctypes.data, len(file))
    staging = MutableBytes(0x1000, need.bytes)  # never touched: every case below fails first
    maps = (TileMapping * need.tiles)()
    for bad_roi in (Roi(0, 0, 0, 5), Roi(250, 0, 51, 5), Roi(0, 199, 5, 2)):
        assert cuda.roi_staging_size(meta, bad_roi)[0] == Status.invalid_roi
        assert cuda.stage_roi_tiles(meta, bad_roi, archive, staging, maps)[0] == \
            Status.invalid_roi
    assert cuda.stage_roi_tiles(meta, roi, ConstBytes(None, len(file)), staging, maps)[0] == \
        Status.invalid_argument
    assert cuda.stage_roi_tiles(meta, roi, ConstBytes(src.ctypes.data, len(file) - 1), staging,
                                maps)[0] == Status.invalid_argument
    assert cuda.stage_roi_tiles(meta, roi, archive, MutableBytes(0x1000, need.bytes - 1),
                                maps)[0] == Status.buffer_too_small
    short = (TileMapping * (need.tiles - 1))()
    assert cuda.stage_roi_tiles(meta, roi, archive, staging, short)[0] == Status.buffer_too_small


def permuted_archive(oracle_lib, frame, tile, seed):
    """The file's tile payloads in a random order after its header and index, and metadata
    (built with ImageMetadata.create) that points at the new places."""
    file = oracle_lib.compress_image(frame, tile)
    st, meta = api.parse_metadata(np.frombuffer(file, dtype=np.uint8))
    assert st == Status.success
    tiles = meta.tiles.copy()
    start = int(tiles["offset"][0])
    order = np.random.default_rng(seed).permutation(len(tiles))
    out = bytearray(file[:start])
    for t in order:
        a, n = int(tiles["offset"][t]), int(tiles["length"][t])
        tiles["offset"][t] = len(out)
        out += file[a:a + n]
    st, moved = api.ImageMetadata.create(meta.image, meta.tile, len(out), tiles,
                                         meta.segments.copy())
    assert st == Status.success
    return bytes(out), moved


def test_out_of_order_payloads_split_runs(oracle_lib):
    """Tiles stored out of file order (possible in metadata a caller builds) start new copies;
    the sizes still follow the tables."""
    frame = workloads.detector_frame(900, 500, seed=8)
    for tile in api.TILE_SHAPES:
        _, meta = permuted_archive(oracle_lib, frame, tile, seed=tile[0])
        for roi in ((0, 0, 900, 500), (100, 40, 333, 210)):
            st, r = cuda.roi_staging_size(meta, Roi(*roi))
            assert st == Status.success
            assert (r.tiles, r.bytes, r.copies) == expected(meta, roi, tile)
            assert r.copies > (roi[1] + roi[3] - 1) // tile[1] - roi[1] // tile[1] + 1
