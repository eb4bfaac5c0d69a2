#pragma once
// Drop-in replacement for the reference's include/tilestream/info.h (info.h:1-10).
#include <string>

namespace tilestream {

[[nodiscard]] const char *version() noexcept;
[[nodiscard]] std::string info_json();

} // namespace tilestream
