// Whole-image decode of .tsc files that were never parsed on the host (extension; no reference
// counterpart).
//
// The reference validates an untrusted file on the host (parse_metadata walks every index entry
// and row descriptor) before its tiles reach the GPU. Here the host checks only each file's
// 64-byte header, with parse_metadata's header rules and statuses, from a host copy of those
// bytes; the decoder validates everything else on the device, tile by tile, with the same rules
// parse_metadata applies: every index entry (mode, reserved bytes, geometry, lengths, payloads
// chained from the end of the index to the end of the file), every RAW and CONSTANT payload's
// padding, and every row descriptor (seed range, width, reserved bytes, packed length, unused
// high bits of a row's last word), and it checks that the device bytes begin with the header
// the host checked. A file accepted by parse_metadata decodes to the same pixels; a file that
// parse_metadata rejects during its walk reports malformed_data in its result record.
//
// There are no host tables, no allocation and no host synchronization: the files travel in the
// decode launch's parameter block, so a call costs the host a header check per file and one
// launch. The decoder's trusted-input machinery (index entries and rows read on the device) does
// the walk, with the rules above added.
#pragma once

#include <tilestream/cuda.h>

#include <cstdint>

namespace tilestream::cuda {

// One file to decode whole.
struct UnparsedFile {
    ConstBytes bytes;       // device memory: the whole file, 4-byte aligned (size = file size)
    const void *header = nullptr; // host memory: a copy of the file's first 64 bytes
    ImageView output;       // device memory: the image's type and size, any valid pitch
};

inline constexpr std::uint64_t max_unparsed_files = 16;

// Enqueues the decode of `count` files (at most max_unparsed_files) on `stream`; results[i]
// receives file i's DeviceResult: success and its pixel bytes, or malformed_data when the
// device walk rejects the file (its output is then unspecified: tiles decoded before the
// failure may have been written). Before anything is enqueued the host returns
// invalid_argument for a null `files`, `header` or result buffer, a misaligned input, result
// buffer or output, or written ranges that overlap anything else (an output with any input,
// output or the result records; the records with any input); resource_limit above
// max_unparsed_files; buffer_too_small when results.count < count; the header statuses of
// parse_metadata (malformed_data, unsupported_format, unsupported_type, size_overflow;
// bytes.size is the file size); invalid_argument for an output whose image is not the file's;
// and the device checks of the plan API (stream and pointers on the current device; a pending
// CUDA error is left for the caller and reported as cuda_error). count 0 enqueues nothing.
[[nodiscard]] Status decode_unparsed_async(const UnparsedFile *files, std::uint64_t count,
                                           ResultBuffer results, cudaStream_t stream) noexcept;

} // namespace tilestream::cuda
