#pragma once
// Drop-in replacement for the reference's include/tilestream/cpu.h (cpu.h:1-14): the scalar
// host codec. Buffers are caller-owned and must not overlap; FP32 samples are bit words.
#include <tilestream/api.h>

namespace tilestream::cpu {

// output.size must be at least compress_bound; on failure nothing is written.
[[nodiscard]] Status compress(ConstImageView input, TileShape tile, MutableBytes output,
                              std::uint64_t &bytes_written) noexcept;
[[nodiscard]] Status decompress(ConstBytes input, ImageView output,
                                const ParseLimits &limits = {}) noexcept;

} // namespace tilestream::cpu
