"""Python mirror of include/tilestream/cpu.h: the scalar host codec of the library."""
from __future__ import annotations

import ctypes as C

from . import _native as N
from .api import ConstBytes, ConstImageView, ImageView, MutableBytes, ParseLimits, Status, TileShape


def compress(input: ConstImageView, tile: TileShape | None, output: MutableBytes):
    """Returns (Status, bytes_written)."""
    written = C.c_uint64(0)
    st = N.lib().ts_cpu_compress(input, tile if tile is not None else TileShape(), output,
                                 C.byref(written))
    return Status(st), written.value


def decompress(input: ConstBytes, output: ImageView, limits: ParseLimits | None = None) -> Status:
    return Status(N.lib().ts_cpu_decompress(input, output,
                                            C.byref(limits) if limits is not None else None))
