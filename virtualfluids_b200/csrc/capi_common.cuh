// capi_common.cuh -- status and error reporting shared by the C entry points.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "../../include/vf_b200.h"

namespace vfb
{
// records a formatted message for vfb_last_error() and returns code
int setError(int code, const char* fmt, ...);
void clearError();
// maps a pending launch error to VFB_ERR_CUDA with the kernel name
int checkLaunch(const char* what);
} // namespace vfb
