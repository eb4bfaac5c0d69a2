"""TIFF import and export (io::read_tiff / io::write_tiff) on the host, in the manner of the
reference tests/tiff_test.cpp:180-420.

Files the library writes are read back by the library and by Pillow's bundled libtiff (an
independent TIFF implementation); strip files that libtiff writes are read by the library. The
cases libtiff cannot be asked for through Pillow (big-endian files, floating-point predictor,
short payloads, unsupported tag values, a second directory) are built here by `make_tiff`, a
small writer of the TIFF 6.0 / BigTIFF container kept in this file as test infrastructure.
"""
import ctypes as C
import os
import struct
import zlib

import numpy as np
import pytest

from tilestream_b200 import _native as N
from tilestream_b200 import api, cpu
from tilestream_b200.api import (PixelType, Status, TiffReadLimits, TiffWriteOptions,
                                 TileShape)

W, H = 33, 17
SPECIAL = [0x00000000, 0x80000000, 0x7f800000, 0xff800000, 0x00000001, 0x80000001,
           0x007fffff, 0x807fffff, 0x7f7fffff, 0xff7fffff, 0x7fc01234, 0x7fa12345,
           0xffc0abcd, 0x3f800000, 0xbf800000, 0x00800000]


def u16_image(w, h):
    y, x = np.mgrid[0:h, 0:w]
    return ((y * 257 + x * 3) & 0xFFFF).astype(np.uint16)


def f32_image(w, h):
    words = (np.uint32(0x3f000000) + np.arange(w * h, dtype=np.uint32))
    words[:len(SPECIAL)] = SPECIAL[:w * h]
    return words.view(np.float32).reshape(h, w)


def same_words(a, b):
    return a.dtype == b.dtype and a.shape == b.shape and \
        np.array_equal(a.view(np.uint8), b.view(np.uint8))


def pillow():
    PIL = pytest.importorskip("PIL")
    from PIL import Image, features
    if not features.check("libtiff"):
        pytest.skip("Pillow without libtiff")
    return Image


# ---- a minimal TIFF container writer (test infrastructure) -------------------------------

SHORT, LONG, LONG8 = 3, 4, 16


def make_tiff(path, blocks, tags, *, big=False, order="<", second=False, counts=None):
    """Writes blocks (bytes) after the header and one directory of `tags` ({tag: (type,
    values)}); the strip or tile offsets (273 or 324) and byte counts (279 or 325) are filled
    from the blocks unless given. second: the directory is written twice, chained."""
    o = order
    head = (b"II" if o == "<" else b"MM") + (
        struct.pack(o + "HHHQ", 43, 8, 0, 0) if big else struct.pack(o + "HI", 42, 0))
    body = bytearray(head)
    offsets = []
    for b in blocks:
        offsets.append(len(body))
        body += b
        if len(body) % 2:
            body += b"\0"
    tags = dict(tags)
    off_tag, cnt_tag = (324, 325) if 322 in tags else (273, 279)
    arr = LONG8 if big else LONG
    tags.setdefault(off_tag, (arr, offsets))
    tags.setdefault(cnt_tag, (arr, counts if counts is not None else [len(b) for b in blocks]))
    fmt = {SHORT: "H", LONG: "I", LONG8: "Q"}
    inline = 8 if big else 4

    def directory(at, next_at):
        # values that do not fit go right after the entries
        n = len(tags)
        entry = 20 if big else 12
        ext = at + (8 if big else 2) + n * entry + (8 if big else 4)
        out, extra = bytearray(struct.pack(o + ("Q" if big else "H"), n)), bytearray()
        for tag in sorted(tags):
            typ, vals = tags[tag]
            raw = b"".join(struct.pack(o + fmt[typ], v) for v in vals)
            if len(raw) <= inline:
                field = raw.ljust(inline, b"\0")
            else:
                field = struct.pack(o + ("Q" if big else "I"), ext + len(extra))
                extra += raw
                if len(extra) % 2:
                    extra += b"\0"
            out += struct.pack(o + ("HHQ" if big else "HHI"), tag, typ, len(vals)) + field
        out += struct.pack(o + ("Q" if big else "I"), next_at)
        return out + extra

    first = len(body)
    d1 = directory(first, 0)
    if second:
        d1 = directory(first, first + len(d1))
        d2 = directory(first + len(d1), 0)
        body += d1 + d2
    else:
        body += d1
    if big:
        body[8:16] = struct.pack(o + "Q", first)
    else:
        body[4:8] = struct.pack(o + "I", first)
    with open(path, "wb") as f:
        f.write(bytes(body))


def base_tags(w, h, bits=16, fmt=1, samples=1, planar=1, orientation=1, photometric=1,
              compression=1, predictor=None, rows=None, tile=None):
    t = {256: (LONG, [w]), 257: (LONG, [h]), 258: (SHORT, [bits] * samples),
         259: (SHORT, [compression]), 262: (SHORT, [photometric]), 274: (SHORT, [orientation]),
         277: (SHORT, [samples]), 284: (SHORT, [planar]), 339: (SHORT, [fmt] * samples)}
    if predictor is not None:
        t[317] = (SHORT, [predictor])
    if rows is not None:
        t[278] = (LONG, [rows])
    if tile is not None:
        t[322] = (LONG, [tile[0]])
        t[323] = (LONG, [tile[1]])
    return t


def strips_of(img, rows, order="<", predictor=1, deflate=False):
    """Strip blocks of a (h, w) array: predictor 2 (horizontal) or 3 (floating point), then
    optional zlib, samples in `order`."""
    h, w = img.shape
    out = []
    for y in range(0, h, rows):
        part = img[y:y + rows]
        if predictor == 3:
            words = part.view(np.uint32 if part.itemsize == 4 else np.uint16)
            b = words.astype(">u4" if part.itemsize == 4 else ">u2").view(np.uint8)
            s = part.itemsize
            planes = b.reshape(part.shape[0], w, s).transpose(0, 2, 1).reshape(part.shape[0], -1)
            planes = planes.astype(np.int16)
            diff = planes.copy()
            diff[:, 1:] = planes[:, 1:] - planes[:, :-1]
            raw = (diff & 0xFF).astype(np.uint8).tobytes()
        else:
            words = part.view(np.uint16 if part.itemsize == 2 else np.uint32).astype(np.int64)
            if predictor == 2:
                d = words.copy()
                d[:, 1:] = words[:, 1:] - words[:, :-1]
                words = d & ((1 << (8 * part.itemsize)) - 1)
            kind = ("u2" if part.itemsize == 2 else "u4")
            raw = words.astype(order + kind).tobytes()
        out.append(zlib.compress(raw) if deflate else raw)
    return out


# ---- C-ABI helpers -----------------------------------------------------------------------

def read_handle(path, limits=None, handle=None):
    """ts_read_tiff through the C entry point; returns (status, handle after the call)."""
    h = C.c_void_p(handle)
    st = N.lib().ts_read_tiff(None if path is None else os.fsencode(path),
                              C.byref(limits) if limits is not None else None, C.byref(h))
    return Status(st), h.value


def pixels_of(handle):
    spec, pitch, data, size = api.ImageSpec(), C.c_uint64(), C.c_void_p(), C.c_uint64()
    assert N.lib().ts_tiff_image_pixels(handle, C.byref(spec), C.byref(pitch), C.byref(data),
                                        C.byref(size)) == 0
    raw = np.ctypeslib.as_array(C.cast(data, C.POINTER(C.c_uint8)), (size.value,)).copy()
    return spec, pitch.value, raw


# ---- tests ---------------------------------------------------------------------------------

CASES = [
    ("u16-none.tif", np.uint16, TiffWriteOptions()),
    ("u16-deflate.tif", np.uint16, TiffWriteOptions(0, 1, 0, 128, 32, 6)),
    ("u16-predictor.tif", np.uint16, TiffWriteOptions(0, 1, 1, 64, 64, 6)),
    ("u16-big.tif", np.uint16, TiffWriteOptions(1, 0, 0, 256, 16, 6)),
    ("f32-none.tif", np.float32, TiffWriteOptions()),
    ("f32-deflate-big.tif", np.float32, TiffWriteOptions(1, 1, 0, 64, 64, 6)),
]


@pytest.mark.parametrize("name,dtype,options", CASES, ids=[c[0] for c in CASES])
def test_tiled_classic_and_bigtiff_round_trip(tmp_path, name, dtype, options):
    """tiff_test.cpp:180-243: written tiled, read back bit for bit, with the compression,
    predictor and signature asked for; libtiff (through Pillow) reads the same words."""
    Image = pillow()
    img = u16_image(W, H) if dtype == np.uint16 else f32_image(W, H)
    path = str(tmp_path / name)
    assert api.write_tiff(path, img, options) == Status.success
    st, got = api.read_tiff(path)
    assert st == Status.success
    assert got["type"] == (PixelType.uint16 if dtype == np.uint16 else PixelType.float32)
    assert (got["width"], got["height"]) == (W, H)
    assert got["pitch_bytes"] == W * img.itemsize
    assert same_words(got["pixels"], img)
    im = Image.open(path)
    tags = dict(im.tag_v2)
    assert 322 in tags and 323 in tags  # tiled
    assert tags[322] == options.tile_width and tags[323] == options.tile_height
    assert tags[259] == (8 if options.compression else 1)
    if options.compression:
        assert tags.get(317, 1) == (2 if options.horizontal_predictor else 1)
    assert same_words(np.array(im), img)
    with open(path, "rb") as f:
        assert f.read(4)[2] == (43 if options.bigtiff else 42)


def test_imports_strips_written_by_libtiff(tmp_path):
    """tiff_test.cpp:245-265: deflate strips (7 rows per strip for uint16, one strip for FP32)
    written by libtiff import to the same words; so do uncompressed strips."""
    Image = pillow()
    w, h = 35, 19
    for img, rows in ((u16_image(w, h), 7), (f32_image(w, h), h)):
        for compression in ("tiff_adobe_deflate", None):
            path = str(tmp_path / f"{img.dtype}-{compression}.tif")
            Image.fromarray(img).save(path, compression=compression, tiffinfo={278: rows})
            st, got = api.read_tiff(path)
            assert st == Status.success, (path, st)
            assert same_words(got["pixels"], img)


def test_tsc_tiff_tsc_preserves_pixels(tmp_path):
    """tiff_test.cpp:267-316: .tsc -> pixels -> TIFF (deflate, predictor for uint16) -> pixels
    -> .tsc gives the same archive bytes."""
    w, h = 129, 33
    for img in (u16_image(w, h), f32_image(w, h)):
        ptype = PixelType.uint16 if img.dtype == np.uint16 else PixelType.float32
        st, bound = api.compress_bound(api.image_spec(ptype, w, h), TileShape(128, 32))
        first = np.zeros(bound, np.uint8)
        st, n1 = cpu.compress(api.const_view(img, ptype, w, h), None, api.mutable_bytes(first))
        assert st == Status.success
        decoded = np.zeros_like(img)
        assert cpu.decompress(api.const_bytes(first, n1),
                              api.view(decoded, ptype, w, h)) == Status.success
        assert same_words(decoded, img)
        path = str(tmp_path / f"{img.dtype}-tsc.tif")
        options = TiffWriteOptions(0, 1, 1 if ptype == PixelType.uint16 else 0, 128, 32, 6)
        assert api.write_tiff(path, decoded, options) == Status.success
        st, got = api.read_tiff(path)
        assert st == Status.success and same_words(got["pixels"], img)
        second = np.zeros(bound, np.uint8)
        st, n2 = cpu.compress(api.const_view(got["pixels"], ptype, w, h), None,
                              api.mutable_bytes(second))
        assert st == Status.success and n2 == n1
        assert np.array_equal(first[:n1], second[:n2])


UNSUPPORTED = [
    ("uint8", dict(bits=8, fmt=1)),
    ("int16", dict(bits=16, fmt=2)),
    ("float64", dict(bits=64, fmt=3)),
    ("rgb", dict(bits=8, fmt=1, samples=3, photometric=2)),
    ("separate", dict(planar=2)),
    ("bottom", dict(orientation=4)),
    ("white", dict(photometric=0)),
    ("multi", dict()),
    ("lzw", dict(compression=5)),
    ("u16-float-predictor", dict(compression=8, predictor=3)),
]


@pytest.mark.parametrize("name,kw", UNSUPPORTED, ids=[c[0] for c in UNSUPPORTED])
def test_rejects_unsupported_tags_without_conversion(tmp_path, name, kw):
    """tiff_test.cpp:318-360: unsupported_format, and the caller's image is not replaced."""
    samples = kw.get("samples", 1)
    nbytes = 2 * 2 * samples * ((kw.get("bits", 16) + 7) // 8)
    block = bytes(nbytes)
    if kw.get("compression") == 8:
        block = zlib.compress(block)
    path = str(tmp_path / f"{name}.tif")
    make_tiff(path, [block], base_tags(2, 2, rows=2, **kw), second=(name == "multi"))
    good = str(tmp_path / "good.tif")
    assert api.write_tiff(good, u16_image(7, 9)) == Status.success
    st, keep = read_handle(good)
    assert st == Status.success
    st, after = read_handle(path, handle=keep)
    assert st == Status.unsupported_format and after == keep
    spec, _, raw = pixels_of(keep)
    assert spec.width == 7 and same_words(raw.view(np.uint16).reshape(9, 7), u16_image(7, 9))
    N.lib().ts_tiff_image_destroy(keep)


def test_limits_and_invalid_arguments(tmp_path):
    """tiff_test.cpp:362-408."""
    img = u16_image(33, 17)
    path = str(tmp_path / "valid.tif")
    assert api.write_tiff(path, img) == Status.success
    big = (1 << 63) - 1
    for limits in (TiffReadLimits(32, 0xFFFFFFFF, big), TiffReadLimits(0xFFFFFFFF, 16, big),
                   TiffReadLimits(0xFFFFFFFF, 0xFFFFFFFF, img.nbytes - 1)):
        assert api.read_tiff(path, limits)[0] == Status.resource_limit
    assert api.read_tiff(path, TiffReadLimits(0xFFFFFFFF, 0xFFFFFFFF, img.nbytes))[0] == \
        Status.success
    assert api.read_tiff(path, TiffReadLimits(0, 1, 1))[0] == Status.invalid_argument
    assert read_handle(None)[0] == Status.invalid_argument
    assert api.read_tiff(str(tmp_path / "missing.tif"))[0] == Status.io_error
    assert N.lib().ts_write_tiff(None, api.const_view(img, PixelType.uint16, 33, 17),
                                 None) == Status.invalid_argument

    def write(name, view, options=None):
        p = str(tmp_path / name)
        st = Status(N.lib().ts_write_tiff(os.fsencode(p), view,
                                          C.byref(options) if options is not None else None))
        return st, os.path.exists(p)

    bad_pitch = api.const_view(img, PixelType.uint16, 33, 17, 65, img.nbytes)
    assert write("bad-pitch.tif", bad_pitch) == (Status.invalid_argument, False)
    v = api.const_view(img, PixelType.uint16, 33, 17)
    assert write("bad-tile.tif", v, TiffWriteOptions(0, 0, 0, 15, 32, 6)) == \
        (Status.invalid_argument, False)
    assert write("bad-predictor.tif", v, TiffWriteOptions(0, 0, 1, 128, 32, 6)) == \
        (Status.invalid_argument, False)
    assert write("bad-level.tif", v, TiffWriteOptions(0, 1, 0, 128, 32, 0)) == \
        (Status.invalid_argument, False)
    assert write("bad-compression.tif", v, TiffWriteOptions(0, 2, 0, 128, 32, 6)) == \
        (Status.invalid_argument, False)
    fimg = f32_image(33, 17)
    assert write("float-predictor.tif", api.const_view(fimg, PixelType.float32, 33, 17),
                 TiffWriteOptions(0, 1, 1, 128, 32, 6)) == (Status.invalid_argument, False)
    side = 1 << 20
    huge = api.ConstImageView(4096, api.image_spec(PixelType.uint16, side, side), side * 2,
                              side * 2 * side)
    assert write("too-many-tiles.tif", huge, TiffWriteOptions(1, 0, 0, 16, 16, 6)) == \
        (Status.size_overflow, False)
    # A directory that does not exist: io_error.
    st = api.write_tiff(str(tmp_path / "no" / "such" / "dir.tif"), img)
    assert st == Status.io_error


@pytest.mark.parametrize("tiled", [False, True])
def test_short_tile_and_strip_are_io_errors(tmp_path, tiled):
    """tiff_test.cpp:410-421: a 16x16 uint16 block stored in 256 bytes."""
    path = str(tmp_path / ("short-tile.tif" if tiled else "short-strip.tif"))
    tags = base_tags(16, 16, tile=(16, 16)) if tiled else base_tags(16, 16, rows=16)
    make_tiff(path, [bytes(256)], tags)
    assert api.read_tiff(path)[0] == Status.io_error
    # The same for a deflate stream that ends early, and one that is not a zlib stream.
    full = zlib.compress(bytes(512))
    for block in (full[:len(full) // 2], b"\x01\x02\x03\x04"):
        make_tiff(path, [block], {**tags, 259: (SHORT, [8])})
        assert api.read_tiff(path)[0] == Status.io_error
    # Offsets past the end of the file.
    make_tiff(path, [bytes(512)], tags, counts=[512 + 4096])
    assert api.read_tiff(path)[0] == Status.io_error


@pytest.mark.parametrize("order", ["<", ">"])
@pytest.mark.parametrize("big", [False, True])
def test_byte_orders_predictors_and_strip_shapes(tmp_path, order, big):
    """Either byte order, classic or BigTIFF, strips of several heights (the last one short),
    no RowsPerStrip (one strip), horizontal predictor on 16- and 32-bit samples and the
    floating-point predictor."""
    w, h = 37, 23
    u, f = u16_image(w, h), f32_image(w, h)
    cases = [(u, 5, 1, False), (u, 23, 2, True), (u, 8, 1, True), (f, 6, 1, False),
             (f, 7, 3, True), (f, 23, 2, True), (u, None, 1, False)]
    for k, (img, rows, pred, deflate) in enumerate(cases):
        bits, fmt = (16, 1) if img.dtype == np.uint16 else (32, 3)
        blocks = strips_of(img, rows or h, order, pred, deflate)
        tags = base_tags(w, h, bits, fmt, rows=rows, compression=8 if deflate else 1,
                         predictor=pred if deflate else None)
        path = str(tmp_path / f"case{k}.tif")
        make_tiff(path, blocks, tags, big=big, order=order)
        st, got = api.read_tiff(path)
        assert st == Status.success, (k, st)
        assert same_words(got["pixels"], img), k


def test_tiles_larger_than_the_image_and_ragged_edges(tmp_path):
    """Tiles cut at the right and bottom edges, and an image smaller than one tile, from the
    library's writer to its reader and to libtiff."""
    Image = pillow()
    for w, h, tw, th in ((1, 1, 16, 16), (17, 1, 16, 16), (300, 70, 128, 32), (16, 16, 16, 16)):
        img = u16_image(w, h)
        path = str(tmp_path / f"t{w}x{h}.tif")
        assert api.write_tiff(path, img, TiffWriteOptions(0, 1, 1, tw, th, 9)) == Status.success
        st, got = api.read_tiff(path)
        assert st == Status.success and same_words(got["pixels"], img)
        assert same_words(np.array(Image.open(path)), img)


def test_c_entry_points_refuse_null_arguments(tmp_path):
    """The C layer's own argument checks: null outputs and handles are invalid_argument, and a
    compression value outside the enum is refused before anything is written."""
    img = u16_image(20, 10)
    path = str(tmp_path / "c.tif")
    assert N.lib().ts_read_tiff(os.fsencode(path), None, None) == Status.invalid_argument
    spec, pitch, data, size = api.ImageSpec(), C.c_uint64(), C.c_void_p(), C.c_uint64()
    assert N.lib().ts_tiff_image_pixels(None, C.byref(spec), C.byref(pitch), C.byref(data),
                                        C.byref(size)) == Status.invalid_argument
    N.lib().ts_tiff_image_destroy(None)  # a no-op
    v = api.const_view(img, PixelType.uint16, 20, 10)
    assert N.lib().ts_write_tiff(os.fsencode(path), v,
                                 C.byref(TiffWriteOptions(0, 7, 0, 128, 32, 6))) == \
        Status.invalid_argument
    assert not os.path.exists(path)
    assert api.write_tiff(path, img) == Status.success
    st, h = read_handle(path)
    assert st == Status.success
    assert N.lib().ts_tiff_image_pixels(h, None, C.byref(pitch), C.byref(data),
                                        C.byref(size)) == Status.invalid_argument
    N.lib().ts_tiff_image_destroy(h)
