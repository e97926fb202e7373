// storage.cuh -- population storage formats.
//
// The stored populations are the shifted deviations f_i - w_i, the variable
// VirtualFluids already stores (its init writes w_i * (drho + ...),
// InitNavierStokesCompressible_Device.cu:175-200).  FP32 and FP64 store them
// as they are.  The precision form stores the same deviations in 16 bits and
// widens them to FP32 for all arithmetic:
//   FP16  IEEE half, multiplied by an exact power of two on store (and by its
//         inverse on load) so that small deviations stay in the normal range;
//   BF16  bfloat16, unscaled (it has the exponent range of FP32);
//   FX16  16-bit fixed point of the deviation relative to its weight:
//         f_i - w_i = q * w_i * 2^-17 with q an int16, so |f_i - w_i| < w_i / 4
//         is held with a uniform step of w_i * 2^-17 (values beyond saturate).
//         At the flows of the benchmarks (|f_i - w_i| / w_i up to 0.16 at
//         u0 = 0.05) this keeps 4 to 6 more significant bits than FP16.
//   FX16W the same int16 code over a range that widens with the number of
//         non-zero components of the direction: f_i - w_i = q * w_i * R * 2^-15
//         with R = 1/4 (rest), 1/2 (faces), 1 (edges and corners), for flows
//         whose deviations leave FX16's quarter of the weight (a bluff body's
//         refined wake reaches 0.39 / 0.55 / 0.72 of the weight on faces /
//         edges / corners); the step of the face populations doubles.
// Every access names the direction d whose slot it touches (the slots of d
// and of its inverse hold populations of equal weight), so a format may scale
// per direction.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdint>

#include "d3q27.cuh"

namespace vfb
{
template <class S>
struct Storage;

template <>
struct Storage<float> {
    using R = float;
    static constexpr int id = 0;
    static constexpr bool scaled = false;
    __device__ __forceinline__ static R load(const float* p, int) { return *p; }
    __device__ __forceinline__ static void store(float* p, R v, int) { *p = v; }
    __device__ __forceinline__ static R loadRaw(const float* p) { return *p; }
    __device__ __forceinline__ static void storeRaw(float* p, R v) { *p = v; }
    static constexpr float invScale(int) { return 1.0f; }
    static constexpr float scale(int) { return 1.0f; }
};

template <>
struct Storage<double> {
    using R = double;
    static constexpr int id = 1;
    static constexpr bool scaled = false;
    __device__ __forceinline__ static R load(const double* p, int) { return *p; }
    __device__ __forceinline__ static void store(double* p, R v, int) { *p = v; }
};

// 2^12: deviations down to ~1.5e-8 stay normal, up to 16 in magnitude fit
constexpr float kHalfScale = 4096.0f;
constexpr float kHalfInvScale = 1.0f / 4096.0f;

template <>
struct Storage<__half> {
    using R = float;
    static constexpr int id = 2;
    static constexpr bool scaled = true;
    // the stored value of a solid node's rest population (the largest finite half)
    static constexpr float marker = 65504.0f;
    static constexpr float invScale(int) { return kHalfInvScale; }
    static constexpr float scale(int) { return kHalfScale; }
    __device__ __forceinline__ static R load(const __half* p, int) { return __half2float(*p) * kHalfInvScale; }
    __device__ __forceinline__ static void store(__half* p, R v, int) { *p = __float2half_rn(v * kHalfScale); }
    // the stored number without the scale (a caller applies invScale(d) /
    // scale(d) itself, e.g. to two values in one paired multiply)
    __device__ __forceinline__ static R loadRaw(const __half* p) { return __half2float(*p); }
    __device__ __forceinline__ static void storeRaw(__half* p, R v) { *p = __float2half_rn(v); }
};

template <>
struct Storage<__nv_bfloat16> {
    using R = float;
    static constexpr int id = 3;
    static constexpr bool scaled = false;
    __device__ __forceinline__ static R load(const __nv_bfloat16* p, int) { return __bfloat162float(*p); }
    __device__ __forceinline__ static void store(__nv_bfloat16* p, R v, int) { *p = __float2bfloat16_rn(v); }
    __device__ __forceinline__ static R loadRaw(const __nv_bfloat16* p) { return __bfloat162float(*p); }
    __device__ __forceinline__ static void storeRaw(__nv_bfloat16* p, R v) { *p = __float2bfloat16_rn(v); }
    static constexpr float invScale(int) { return 1.0f; }
    static constexpr float scale(int) { return 1.0f; }
};

// 2^17 / w_d for the four weight classes: 27/8, 27/2, 54 and 216 times 2^17,
// all exact in FP32
__host__ __device__ constexpr float fx16Scale(int d)
{
    return order(d) == 0 ? 442368.0f : order(d) == 1 ? 1769472.0f : order(d) == 2 ? 7077888.0f : 28311552.0f;
}

template <>
struct Storage<int16_t> {
    using R = float;
    static constexpr int id = 4;
    static constexpr bool scaled = true;
    // the stored value of a solid node's rest population (the saturated code)
    static constexpr float marker = 32767.0f;
    static constexpr float invScale(int d) { return 1.0f / fx16Scale(d); }
    static constexpr float scale(int d) { return fx16Scale(d); }
    __device__ __forceinline__ static R loadRaw(const int16_t* p)
    {
        float r;
        asm("cvt.rn.f32.s16 %0, %1;" : "=f"(r) : "h"(*p));
        return r;
    }
    // round to nearest even, saturating at the ends of the int16 range
    __device__ __forceinline__ static void storeRaw(int16_t* p, R v)
    {
        int16_t q;
        asm("cvt.rni.sat.s16.f32 %0, %1;" : "=h"(q) : "f"(v));
        *p = q;
    }
    __device__ __forceinline__ static R load(const int16_t* p, int d) { return loadRaw(p) * invScale(d); }
    __device__ __forceinline__ static void store(int16_t* p, R v, int d) { storeRaw(p, v * scale(d)); }
};

// FX16W: an int16 code whose scale is 2^15 / (R_d w_d) (storage.cuh header)
struct fx16w_t {
    int16_t q;
};

// 2^15 / (R_d w_d) for the four weight classes: 27/2, 27, 54 and 216 times
// 2^15, all exact in FP32
__host__ __device__ constexpr float fx16wScale(int d)
{
    return order(d) == 0 ? 442368.0f : order(d) == 1 ? 884736.0f : order(d) == 2 ? 1769472.0f : 7077888.0f;
}

template <>
struct Storage<fx16w_t> {
    using R = float;
    static constexpr int id = 5;
    static constexpr bool scaled = true;
    static constexpr float marker = 32767.0f;
    static constexpr float invScale(int d) { return 1.0f / fx16wScale(d); }
    static constexpr float scale(int d) { return fx16wScale(d); }
    __device__ __forceinline__ static R loadRaw(const fx16w_t* p)
    {
        float r;
        asm("cvt.rn.f32.s16 %0, %1;" : "=f"(r) : "h"(p->q));
        return r;
    }
    __device__ __forceinline__ static void storeRaw(fx16w_t* p, R v)
    {
        int16_t q;
        asm("cvt.rni.sat.s16.f32 %0, %1;" : "=h"(q) : "f"(v));
        p->q = q;
    }
    __device__ __forceinline__ static R load(const fx16w_t* p, int d) { return loadRaw(p) * invScale(d); }
    __device__ __forceinline__ static void store(fx16w_t* p, R v, int d) { storeRaw(p, v * scale(d)); }
};
} // namespace vfb
