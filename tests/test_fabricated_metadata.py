"""Fabricated host metadata, checked on the host: preparation must reject it, or every tile task
it plans must stay inside the declared buffers.

This is the campaign of the reference's tests/cuda_robustness_test.cpp:245-306
(FabricatedMetadataIsRejectedOrStaysInBounds) with the same engine, seed and draw order: for
uint16 and FP32, a 300x192 image of constant, smooth and noisy bands (all three tile modes) is
encoded with each tile shape, parsed, and 500 times given one fabricated change (one field of
one tile or row record, the file size, or a dropped record) and a random ROI. The reference runs
each accepted plan on the GPU and relies on a memory checker; here the plan is never launched.
ts_inspect_decode runs the host half of prepare_batch (every check that needs no device) and
reports each task's staged bytes and written bytes, which must lie inside the source and output
buffers, with the stage, row-table and tile-size limits of the decoder. The same 3,000 cases are
then safe for the reference suite's own GPU run.
"""
import numpy as np

from tilestream_b200 import api, cuda
from tilestream_b200.api import BatchItem, ConstBytes, Status, TileShape

SOURCE = 0x7f0000000000  # stand-in device addresses: inspection dereferences nothing
OUTPUT = 0x7e0000000000
SHAPES = ((128, 32), (64, 64), (256, 16))
STAGE = {1: 8192, 2: 16384}  # largest tile payload the decoder stages, per pixel type


def mixed_image(o, ptype):
    """tests/cuda_robustness_test.cpp:180-190: bands of 64 rows with the robustness patterns
    0 (constant), 5 (smooth) and 4 (noise), seeds 0, 1, 2; rows are unpadded."""
    s = api.sample_bytes(ptype)
    pitch = 300 * s
    image = np.full(pitch * 192, 0x5A, np.uint8)
    for band, pattern in enumerate((0, 5, 4)):
        image[band * 64 * pitch:(band + 1) * 64 * pitch] = o.fill(ptype, 300, 64, pattern, band,
                                                                  pitch)
    return image, pitch


def cpu_encode(image, ptype, pitch, shape):
    st, bound = api.compress_bound(api.image_spec(ptype, 300, 192), TileShape(*shape))
    out = np.zeros(bound, np.uint8)
    from tilestream_b200 import cpu
    st, written = cpu.compress(api.const_view(image, ptype, 300, 192, pitch),
                               TileShape(*shape), api.mutable_bytes(out))
    assert st == Status.success
    return out[:written].tobytes()


def test_fabricated_metadata_is_rejected_or_stays_in_bounds(oracle_lib):
    engine = oracle_lib.engine(4242)
    statuses = {}
    accepted = tasks_checked = 0
    allowed = {Status.malformed_data, Status.unsupported_format, Status.buffer_too_small}
    for ptype in (1, 2):
        image, pitch = mixed_image(oracle_lib, ptype)
        s = api.sample_bytes(ptype)
        out_pitch = 301 * s  # one padding sample per row, as the reference's Output
        out_capacity = out_pitch * 192
        for shape in SHAPES:
            file = cpu_encode(image, ptype, pitch, shape)
            st, meta = api.parse_metadata(np.frombuffer(file, np.uint8))
            assert st == Status.success
            modes = np.bincount(meta.tiles["mode"], minlength=3)
            assert modes[0] > 0 and modes[1] > 0 and modes[2] > 0, modes
            tiles, segments, file_bytes = meta.tiles, meta.segments, meta.file_bytes
            for _ in range(500):
                t, g, fb = oracle_lib.fabricate(engine, tiles, segments, file_bytes)
                x = engine.next() % 300
                y = engine.next() % 192
                w = 1 + engine.next() % (300 - x)
                h = 1 + engine.next() % (192 - y)
                st, fabricated = api.ImageMetadata.create(meta.image, meta.tile, fb, t, g)
                assert st == Status.success
                item = BatchItem()
                item.compressed_input.bytes = ConstBytes(SOURCE, len(file))
                item.compressed_input.metadata = fabricated.handle
                item.roi = api.Roi(x, y, w, h)
                item.output = api.ImageView(OUTPUT, api.image_spec(ptype, w, h), out_pitch,
                                            out_capacity)
                st, spans = cuda.inspect_decode(cuda.make_request(cuda.Operation.decode_roi,
                                                                  [item]))
                statuses[int(st)] = statuses.get(int(st), 0) + 1
                if st != Status.success:
                    assert st in allowed, st
                    continue
                accepted += 1
                assert len(spans) > 0
                for sp in spans:
                    assert SOURCE <= sp.read_begin < sp.read_end <= SOURCE + len(file)
                    staged = sp.read_end - sp.read_begin
                    assert staged % 4 == 0 and staged <= STAGE[ptype]
                    assert sp.rows_end <= staged
                    assert 1 <= sp.width <= 256 and 1 <= sp.height <= 64
                    if sp.mode == int(api.TileMode.predict_bitpack):
                        assert sp.rows_end >= 8
                    assert OUTPUT <= sp.write_begin < sp.write_end <= OUTPUT + out_capacity
                    tasks_checked += 1
    assert sum(statuses.values()) == 3000
    assert accepted > 0 and statuses.get(int(Status.malformed_data), 0) > 0, statuses
    assert tasks_checked > accepted
