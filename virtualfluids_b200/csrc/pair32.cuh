// pair32.cuh -- two FP32 lattice nodes in one register pair.
//
// sm_100 executes paired FP32 add / multiply / fused multiply-add
// (__fadd2_rn, __fmul2_rn, __ffma2_rn) at the rate of one scalar instruction,
// so the collision of two nodes written with this type issues about half the
// arithmetic instructions of two scalar collisions.  Every paired operation
// rounds each half as the scalar IEEE operation does; divisions and absolute
// values stay scalar per half.  Used for the FP32-arithmetic kernels (FP32,
// FP16 and BF16 storage).
#pragma once

#include <cuda_runtime.h>

#include "collision_math.cuh"

namespace vfb
{

struct F2 {
    float2 v;
    F2() = default;
    __host__ __device__ __forceinline__ F2(float s) : v(make_float2(s, s)) {}
    __host__ __device__ __forceinline__ F2(float a, float b) : v(make_float2(a, b)) {}
};

template <>
struct ScalarOf<F2> {
    using type = float;
};

#ifdef __CUDACC__
__device__ __forceinline__ F2 pairOf(float2 x)
{
    F2 r;
    r.v = x;
    return r;
}
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return pairOf(__fadd2_rn(a.v, b.v)); }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return pairOf(__fmul2_rn(a.v, b.v)); }
// negation and subtraction as one paired multiply / multiply-add by -1 (exact)
__device__ __forceinline__ F2 operator-(F2 a) { return pairOf(__fmul2_rn(a.v, make_float2(-1.0f, -1.0f))); }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return pairOf(__ffma2_rn(b.v, make_float2(-1.0f, -1.0f), a.v)); }
__device__ __forceinline__ F2 operator/(F2 a, F2 b) { return pairOf(make_float2(a.v.x / b.v.x, a.v.y / b.v.y)); }
__device__ __forceinline__ F2& operator+=(F2& a, F2 b)
{
    a = a + b;
    return a;
}
__device__ __forceinline__ F2& operator-=(F2& a, F2 b)
{
    a = a - b;
    return a;
}
__device__ __forceinline__ F2 fma(F2 a, F2 b, F2 c) { return pairOf(__ffma2_rn(a.v, b.v, c.v)); }
__device__ __forceinline__ F2 fabs(F2 a) { return pairOf(make_float2(fabsf(a.v.x), fabsf(a.v.y))); }

#ifdef __CUDA_ARCH__
template <>
__device__ __forceinline__ F2 limiterQuotient<F2>(F2 x, F2 y)
{
    return pairOf(make_float2(__fdividef(x.v.x, y.v.x), __fdividef(x.v.y, y.v.y)));
}
#endif
#endif

// K17 rates of a launch duplicated into both halves
inline K17Rates<F2> pairRates(const K17Rates<float>& r)
{
    K17Rates<F2> p;
    p.omega = F2(r.omega);
    p.OxyyPxzz = F2(r.OxyyPxzz);
    p.OxyyMxzz = F2(r.OxyyMxzz);
    p.Oxyz = F2(r.Oxyz);
    p.oneMinusOxyyPxzz = F2(r.oneMinusOxyyPxzz);
    p.oneMinusOxyyMxzz = F2(r.oneMinusOxyyMxzz);
    p.oneMinusOxyz = F2(r.oneMinusOxyz);
    p.factorA = F2(r.factorA);
    p.factorB = F2(r.factorB);
    p.minusTau = F2(r.minusTau);
    p.halfMinusOmega = F2(r.halfMinusOmega);
    p.omegaThreeHalves = F2(r.omegaThreeHalves);
    p.minusThreeOmega = F2(r.minusThreeOmega);
    p.secondOrderCorrection = F2(r.secondOrderCorrection);
    p.qlP = F2(r.qlP);
    p.qlM = F2(r.qlM);
    p.qlD = F2(r.qlD);
    p.fourthA = F2(r.fourthA);
    p.fourthB = F2(r.fourthB);
    return p;
}

} // namespace vfb
