// bc_math.cuh -- per-node formulas of the post-collision boundary conditions,
// shared by the BC kernels (bc.cu) and their adjoints (adjoint.cu) so that
// both run the same arithmetic.  Formulas: KernelUtilities.h:171-195 and the
// plain macroscopic sums of NoSlipInterpolatedCompressible.cu:144-160.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "d3q27.cuh"

namespace vfb
{

// directions in the order the reference's BC kernels visit them
__host__ __device__ constexpr int qOrder(int j)
{
    constexpr int t[26] = { dP00, dM00, d0P0, d0M0, d00P, d00M, dPP0, dMM0, dPM0, dMP0, dP0P, dM0M, dP0M,
                            dM0P, d0PP, d0MM, d0PM, d0MP, dPPP, dMMM, dPPM, dMMP, dPMP, dMPM, dPMM, dMPP };
    return t[j];
}

template <class R>
struct BcLattice {
    unsigned long long N;
    const uint32_t* __restrict__ nX;
    const uint32_t* __restrict__ nY;
    const uint32_t* __restrict__ nZ;
    R omega;
};

// drho and velocity from post-collision populations with the plain sums of
// NoSlipInterpolatedCompressible.cu:144-160 (g[d] moves in direction d)
template <class R>
__device__ __forceinline__ void bcMacros(const R* g, R& drho, R& vx1, R& vx2, R& vx3)
{
    R s = g[dPMP];
    s = s + g[dMPP];
    s = s + g[dPPP];
    s = s + g[dMMP];
    s = s + g[dPMM];
    s = s + g[dMPM];
    s = s + g[dPPM];
    s = s + g[dMMM];
    s = s + g[d0PM];
    s = s + g[d0MP];
    s = s + g[d0PP];
    s = s + g[d0MM];
    s = s + g[dP0M];
    s = s + g[dM0P];
    s = s + g[dP0P];
    s = s + g[dM0M];
    s = s + g[dPM0];
    s = s + g[dMP0];
    s = s + g[dPP0];
    s = s + g[dMM0];
    s = s + g[d00P];
    s = s + g[d00M];
    s = s + g[d0P0];
    s = s + g[d0M0];
    s = s + g[dP00];
    s = s + g[dM00];
    s = s + g[d000];
    drho = s;
    const R r1 = R(1) + s;
    vx1 = (((g[dPMP] - g[dMPM]) - (g[dMPP] - g[dPMM])) + ((g[dPPP] - g[dMMM]) - (g[dMMP] - g[dPPM])) +
           ((g[dP0M] - g[dM0P]) + (g[dP0P] - g[dM0M])) + ((g[dPM0] - g[dMP0]) + (g[dPP0] - g[dMM0])) +
           (g[dP00] - g[dM00])) /
          r1;
    vx2 = ((-(g[dPMP] - g[dMPM]) + (g[dMPP] - g[dPMM])) + ((g[dPPP] - g[dMMM]) - (g[dMMP] - g[dPPM])) +
           ((g[d0PM] - g[d0MP]) + (g[d0PP] - g[d0MM])) + (-(g[dPM0] - g[dMP0]) + (g[dPP0] - g[dMM0])) +
           (g[d0P0] - g[d0M0])) /
          r1;
    vx3 = (((g[dPMP] - g[dMPM]) + (g[dMPP] - g[dPMM])) + ((g[dPPP] - g[dMMM]) + (g[dMMP] - g[dPPM])) +
           (-(g[d0PM] - g[d0MP]) + (g[d0PP] - g[d0MM])) + ((g[dP0P] - g[dM0M]) - (g[dP0M] - g[dM0P])) +
           (g[d00P] - g[d00M])) /
          r1;
}

// KernelUtilities.h:171-174
template <class R>
__device__ __forceinline__ R feqBC(R drho, R vel, R cuSq, R w)
{
    return w * (drho + R(9) / R(2) * vel * vel * (R(1) + drho) - cuSq);
}

// KernelUtilities.h:189-195
template <class R>
__device__ __forceinline__ R interpNoSlip(R q, R f, R finv, R feq, R omega)
{
    return (R(1) - q) / (R(1) + q) * (f - finv + (f + finv - R(2) * feq * omega) / (R(1) - omega)) * (R(1) / R(2)) +
           (q * (f + finv)) / (R(1) + q);
}

// KernelUtilities.h:176-182
template <class R>
__device__ __forceinline__ R interpVelocity(R q, R f, R finv, R feq, R omega, R vel, R w)
{
    return (R(1) - q) / (R(1) + q) * (f - finv + (f + finv - R(2) * feq * omega) / (R(1) - omega)) * (R(1) / R(2)) +
           (q * (f + finv) - R(6) * w * vel) / (R(1) + q);
}

// KernelUtilities.h:199-206 (the interpolated no-slip value minus w drho)
template <class R>
__device__ __forceinline__ R interpNoSlipPressure(R q, R f, R finv, R feq, R omega, R drho, R w)
{
    return interpNoSlip(q, f, finv, feq, omega) - w * drho;
}

// The wall model's clip (iMEM.cuh:131-136): -3 F forceFactor formed in
// double (the reference's literal 3.0 promotes it), bounded by +-clip with
// the NaN-ignoring double min / max.
template <class R>
__device__ __forceinline__ R imemClip(R clip, R F, R forceFactor)
{
    const double t = -3.0 * (double)F * (double)forceFactor;
    return (R)(clip > -clip ? fmin((double)clip, fmax((double)-clip, t)) : fmax((double)clip, fmin((double)-clip, t)));
}

// one step of a temporal filter, eps v + (1 - eps) mean with the second
// product in double as the reference writes it (iMEM.cuh:78-90)
template <class R>
__device__ __forceinline__ R imemFilter(R eps, R v, R mean)
{
    return (R)((double)(eps * v) + (1.0 - (double)eps) * (double)mean);
}

// The iMEM wall model of one BC entry (iMEM.cuh:57-137, Asmuth et al. 2021):
// the filtered velocities at the sampling node (el, in/out) and at the wall
// node (wm, in/out), the friction velocity u* = kappa |u_el,t| / ln(z / z0)
// at z = samplingOffset + q, the wall shear stress u*^2 along the wall node's
// tangential velocity over the filtered one's magnitude, minus the tangential
// momentum the bounce-back exchanged with the wall at rest (mom), and the wall
// velocity -3 F forceFactor clipped to twice the filtered tangential velocity.
template <class R>
__device__ __forceinline__ void imemWallVelocity(const R n[3], R el[3], R wm[3], const R vw[3], R rho, R z, R z0,
                                                 R forceFactor, const R mom[3], R& uStar, R V[3])
{
    const R dEl = el[0] * n[0] + el[1] * n[1] + el[2] * n[2];
    R t[3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
        t[a] = el[a] - dEl * n[a];
    const R magEl = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
    const R dWm = wm[0] * n[0] + wm[1] * n[1] + wm[2] * n[2];
    R tm[3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
        tm[a] = wm[a] - dWm * n[a];
    const R magWm = sqrt(tm[0] * tm[0] + tm[1] * tm[1] + tm[2] * tm[2]);
    const R dW = vw[0] * n[0] + vw[1] * n[1] + vw[2] * n[2];
    uStar = magEl * R(0.4) / log(z / z0);
    const R tauW = uStar * uStar;
    const R dM = mom[0] * n[0] + mom[1] * n[1] + mom[2] * n[2];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const R Fw = (tauW * R(1)) * ((vw[a] - dW * n[a]) / magWm);
        const R F = Fw - (mom[a] - dM * n[a]) / rho;
        V[a] = imemClip(R(2) * t[a], F, forceFactor);
    }
}

} // namespace vfb
