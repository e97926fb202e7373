// capi_common.cu -- error state of the C ABI (one message per host thread).
#include <cstdarg>
#include <cstdio>

#include "capi_common.cuh"

namespace vfb
{
static thread_local char g_lastError[512] = { 0 };

int setError(int code, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(g_lastError, sizeof(g_lastError), fmt, ap);
    va_end(ap);
    return code;
}

void clearError() { g_lastError[0] = 0; }

int checkLaunch(const char* what)
{
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return setError(VFB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return VFB_OK;
}
} // namespace vfb

extern "C" int vfb_version(void) { return 100; }

extern "C" const char* vfb_last_error(void) { return vfb::g_lastError; }

extern "C" int vfb_storage_bytes(int storage)
{
    switch (storage) {
    case VFB_FP32: return 4;
    case VFB_FP64: return 8;
    case VFB_FP16: return 2;
    case VFB_FX16: return 2;
    case VFB_FX16W: return 2;
    case VFB_BF16: return 2;
    default: return 0;
    }
}

extern "C" int vfb_copy_device_to_host(void* dst, const void* src, size_t bytes, void* stream)
{
    vfb::clearError();
    if (bytes == 0)
        return VFB_OK;
    if (!dst || !src)
        return vfb::setError(VFB_ERR_INVALID_ARGUMENT, "NULL pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
        return vfb::setError(VFB_ERR_CUDA, "device to host copy failed: %s", cudaGetErrorString(cudaGetLastError()));
    return VFB_OK;
}
