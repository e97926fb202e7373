// storage.cuh -- population storage formats.
//
// The stored populations are the shifted deviations f_i - w_i, the variable
// VirtualFluids already stores (its init writes w_i * (drho + ...),
// InitNavierStokesCompressible_Device.cu:175-200).  FP32 and FP64 store them
// as they are.  The precision form stores the same deviations narrowed to
// FP16 or BF16 and widens them to FP32 for all arithmetic.  FP16 multiplies by
// an exact power of two on store (and by its inverse on load) so that small
// deviations stay in the normal range of the format; BF16 has the exponent
// range of FP32 and is stored unscaled.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace vfb
{
template <class S>
struct Storage;

template <>
struct Storage<float> {
    using R = float;
    static constexpr int id = 0;
    static constexpr bool scaled = false;
    __device__ __forceinline__ static R load(const float* p) { return *p; }
    __device__ __forceinline__ static void store(float* p, R v) { *p = v; }
    __device__ __forceinline__ static R loadRaw(const float* p) { return *p; }
    __device__ __forceinline__ static void storeRaw(float* p, R v) { *p = v; }
};

template <>
struct Storage<double> {
    using R = double;
    static constexpr int id = 1;
    static constexpr bool scaled = false;
    __device__ __forceinline__ static R load(const double* p) { return *p; }
    __device__ __forceinline__ static void store(double* p, R v) { *p = v; }
};

// 2^12: deviations down to ~1.5e-8 stay normal, up to 16 in magnitude fit
constexpr float kHalfScale = 4096.0f;
constexpr float kHalfInvScale = 1.0f / 4096.0f;

template <>
struct Storage<__half> {
    using R = float;
    static constexpr int id = 2;
    static constexpr bool scaled = true;
    __device__ __forceinline__ static R load(const __half* p) { return __half2float(*p) * kHalfInvScale; }
    __device__ __forceinline__ static void store(__half* p, R v) { *p = __float2half_rn(v * kHalfScale); }
    // the stored number without the scale (a caller applies kHalfInvScale /
    // kHalfScale itself, e.g. to two values in one paired multiply)
    __device__ __forceinline__ static R loadRaw(const __half* p) { return __half2float(*p); }
    __device__ __forceinline__ static void storeRaw(__half* p, R v) { *p = __float2half_rn(v); }
};

template <>
struct Storage<__nv_bfloat16> {
    using R = float;
    static constexpr int id = 3;
    static constexpr bool scaled = false;
    __device__ __forceinline__ static R load(const __nv_bfloat16* p) { return __bfloat162float(*p); }
    __device__ __forceinline__ static void store(__nv_bfloat16* p, R v) { *p = __float2bfloat16_rn(v); }
    __device__ __forceinline__ static R loadRaw(const __nv_bfloat16* p) { return __bfloat162float(*p); }
    __device__ __forceinline__ static void storeRaw(__nv_bfloat16* p, R v) { *p = __float2bfloat16_rn(v); }
};
} // namespace vfb
