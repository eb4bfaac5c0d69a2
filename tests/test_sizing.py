"""Sizing entry points (include/tilestream/sizing.h) against the reference's own sizing code
(oracle/_ref, built from the reference sources), status and value, over a grid of valid,
boundary and invalid inputs: pixel types, zero and extreme dimensions, unsupported tile
shapes, pitches around the row size, and workspace specs at and past the window limits."""
import itertools

from tilestream_b200 import api
from tilestream_b200.api import ImageSpec, TileShape, WorkspaceSpec

TYPES = (0, 1, 2, 3)
DIMS = (0, 1, 31, 32, 127, 128, 129, 4095, 4096, 65535, 65536, 1 << 31, (1 << 32) - 1)
TILES = ((128, 32), (64, 64), (256, 16), (0, 0), (32, 128), (128, 128), (1, 1), (64, 32))


def test_compress_bound_matches_reference(reference):
    n = 0
    for t, w, h, tile in itertools.product(TYPES, DIMS, DIMS, TILES):
        want = reference.compress_bound(t, w, h, tile)
        st, got = api.compress_bound(ImageSpec(t, w, h), TileShape(*tile))
        assert int(st) == want[0], (t, w, h, tile)
        if want[0] == 0:
            assert got == want[1], (t, w, h, tile)
        n += 1
    assert n == len(TYPES) * len(DIMS) ** 2 * len(TILES)


def test_image_span_matches_reference(reference):
    for t, w, h in itertools.product(TYPES, DIMS, DIMS):
        s = 4 if t == 2 else 2
        for pitch in (0, w * s - 1 if w else 0, w * s, w * s + 1, w * s + 64, (1 << 64) - 1):
            pitch = max(0, min(pitch, (1 << 64) - 1))
            want = reference.image_span(t, w, h, pitch)
            st, got = api.image_span(ImageSpec(t, w, h), pitch)
            assert int(st) == want[0], (t, w, h, pitch)
            if want[0] == 0:
                assert got == want[1], (t, w, h, pitch)


def test_workspace_size_matches_reference(reference):
    images = (0, 1, 2, 4095, 4096, 4097, 1 << 32)
    tiles = (0, 1, 2, 4095, 4096, 4097, 1 << 20, 1 << 40)
    temps = (0, 1, 255, 256, 1 << 40, (1 << 64) - 1)
    for i, k, tile, temp in itertools.product(images, tiles, TILES, temps):
        want = reference.workspace_size(i, k, tile, temp)
        st, got = api.workspace_size(WorkspaceSpec(i, k, TileShape(*tile), temp))
        assert int(st) == want[0], (i, k, tile, temp)
        if want[0] == 0:
            assert got == want[1], (i, k, tile, temp)


def test_documented_examples():
    """The reference's worked examples, independent of the reference build: compress_bound of
    a 1x1 image of either type is 100 B, of a 128x32 uint16 image 8288 B and of 129x33 8708 B
    (docs/format.md:132); the fixed workspace regions for one default tile and one image total
    17664 B, with A256(S) appended, and the empty spec needs zero bytes (docs/api.md:107)."""
    for ptype, w, h, want in ((1, 1, 1, 100), (2, 1, 1, 100), (1, 128, 32, 8288),
                              (1, 129, 33, 8708)):
        st, got = api.compress_bound(ImageSpec(ptype, w, h), TileShape())
        assert int(st) == 0 and got == want, (ptype, w, h)
    for temp, want in ((0, 17664), (1, 17664 + 256), (256, 17664 + 256), (257, 17664 + 512)):
        st, got = api.workspace_size(WorkspaceSpec(1, 1, TileShape(128, 32), temp))
        assert int(st) == 0 and got == want, temp
    st, got = api.workspace_size(WorkspaceSpec(0, 0, TileShape(128, 32), 0))
    assert int(st) == 0 and got == 0
