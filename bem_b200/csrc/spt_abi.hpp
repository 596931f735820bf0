// Error reporting shared by the translation units that define entry points
// of include/spt_b200.h: `fail` records a message for spt_last_error() (per
// host thread) and returns `code`; `cuda_check` turns a CUDA runtime error
// into SPT_ERR_CUDA with the runtime's message.
#pragma once
#include <cuda_runtime.h>

namespace spt_abi {
int fail(int code, const char* fmt, ...);
int cuda_check(cudaError_t e, const char* what);
}  // namespace spt_abi
