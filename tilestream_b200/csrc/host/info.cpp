// version() and info_json() of include/tilestream/info.h: the library version and a small JSON
// report of the CUDA environment (reference: src/info.cpp, diagnostics only).
#include <tilestream/build_config.h>
#include <tilestream/info.h>

#include <cuda_runtime_api.h>

#include <cstdio>
#include <string>

namespace tilestream {

const char *version() noexcept {
    return TILESTREAM_VERSION;
}

std::string info_json() {
    std::string out = "{\"library\":\"tilestream_b200\",\"version\":\"";
    out += version();
    out += "\",\"format\":\"1.0\",\"cuda_arch\":\"sm_100a\"";
    int runtime = 0, driver = 0, count = 0;
    cudaRuntimeGetVersion(&runtime);
    cudaDriverGetVersion(&driver);
    char buf[512];
    std::snprintf(buf, sizeof(buf), ",\"cuda_runtime\":%d,\"cuda_driver\":%d", runtime, driver);
    out += buf;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        static_cast<void>(cudaGetLastError());
        count = 0;
    }
    out += ",\"devices\":[";
    for (int i = 0; i < count; ++i) {
        cudaDeviceProp p{};
        if (cudaGetDeviceProperties(&p, i) != cudaSuccess) {
            static_cast<void>(cudaGetLastError());
            continue;
        }
        std::snprintf(buf, sizeof(buf),
                      "%s{\"index\":%d,\"name\":\"%s\",\"cc\":\"%d.%d\",\"sms\":%d,"
                      "\"memory_bytes\":%zu}",
                      i ? "," : "", i, p.name, p.major, p.minor, p.multiProcessorCount,
                      p.totalGlobalMem);
        out += buf;
    }
    out += "]}";
    return out;
}

} // namespace tilestream
