// Handle accessors shared between the library's translation units (not exported).
#pragma once
#include <cuda_runtime.h>

#include "../../include/dd_gpu.h"
#include "kernels.cuh"

namespace ddk {
IndexView internal_view(dd_index* h);
cudaStream_t internal_stream(dd_index* h);
int internal_device(dd_index* h);
int internal_fail(dd_index* h, int code, const char* msg);
int internal_check_error_word(dd_index* h);
}  // namespace ddk
