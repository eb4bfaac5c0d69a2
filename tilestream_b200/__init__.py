"""TileStream on B200: a B200-native (sm_100a) implementation of TileStream's GPU codec path.

The library is libtilestream_b200.so (C++17 host code + hand-written CUDA kernels) behind the
reference's C++ API (include/tilestream/) and a flat C ABI (include/tilestream_c.h). This package
is the Python view of that ABI, used by the tests and the benchmark:

    from tilestream_b200 import api, cpu, cuda
"""
from . import api, cpu, cuda  # noqa: F401
from .api import (PixelType, Status, TileMode, TileShape, compress_bound, image_span,  # noqa
                  parse_metadata, workspace_size)
