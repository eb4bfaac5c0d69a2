#pragma once
// This library is always built with its CUDA path (sm_100a); the reference generates this
// header from cmake/build_config.h.in.
#define TILESTREAM_WITH_CUDA 1
#define TILESTREAM_VERSION "0.1.0-b200"
