// collision_math.cuh -- per-node collision operators, held in registers.
//
// K17: the compressible cumulant collision of VirtualFluids
// (src/lbm/collision/K17CompressibleNavierStokes.h:87-591, TurbulenceModel::None),
// based on Geier et al., J. Comput. Phys. 348 (2017) 862-888 and 889-898.
// The arithmetic of every retained term is performed in the same order as the
// reference so that FP64 results agree to rounding (FMA contraction aside).
// Two things are different by construction, neither changes a result:
//   * rates that depend only on omega and the limiters are formed once per
//     launch on the host (K17Rates) with the reference's expressions;
//   * cumulants whose post-collision value does not depend on their
//     pre-collision value (orders 4..6 with O4 = O5 = O6 = 1) are never
//     formed: the reference computes them and then multiplies them by
//     (1 - 1) = 0 or cancels them exactly (x + 1 * (-x) = +0).
//
// BGK: src/gpu/core/Kernel/Compressible/NavierStokes/B92/B92CompressibleNavierStokes_Device.cu:194-234.
#pragma once

#include "d3q27.cuh"

namespace vfb
{

// Per-launch constants of the K17 collision (K17CompressibleNavierStokes.h:245-273,
// limiter inputs :176-178, force factor RunCollision.cuh:111-113).
template <class R>
struct K17Rates {
    R omega;
    R OxyyPxzz, OxyyMxzz, Oxyz;       // third-order rates
    R oneMinusOxyyPxzz, oneMinusOxyyMxzz, oneMinusOxyz;
    R factorA, factorB;               // fourth-order modified equilibrium
    R minusTau;                       // -O4 * (1/omega - 1/2)
    R halfMinusOmega;                 // 1/2 * (-omega)
    R omegaThreeHalves;               // omega * 3/2
    R minusThreeOmega;                // -3 * omega
    R secondOrderCorrection;          // 3 * (1 + 1/2 * (-omega))
    R qlP, qlM, qlD;                  // quartic limiters
};

template <class R>
inline K17Rates<R> makeK17Rates(R omega, R qlP, R qlM, R qlD)
{
    K17Rates<R> r;
    r.omega = omega;
    r.OxyyPxzz = R(8) * (-R(2) + omega) * (R(1) + R(2) * omega) / (-R(8) - R(14) * omega + R(7) * omega * omega);
    r.OxyyMxzz = R(8) * (-R(2) + omega) * (-R(7) + R(4) * omega) / (R(56) - R(50) * omega + R(9) * omega * omega);
    r.Oxyz = R(24) * (-R(2) + omega) * (-R(2) - R(7) * omega + R(3) * omega * omega) /
             (R(48) + R(152) * omega - R(130) * omega * omega + R(29) * omega * omega * omega);
    r.oneMinusOxyyPxzz = R(1) - r.OxyyPxzz;
    r.oneMinusOxyyMxzz = R(1) - r.OxyyMxzz;
    r.oneMinusOxyz = R(1) - r.Oxyz;
    r.factorA = (R(4) + R(2) * omega - R(3) * omega * omega) / (R(2) - R(7) * omega + R(5) * omega * omega);
    r.factorB = (R(4) + R(28) * omega - R(14) * omega * omega) / (R(6) - R(21) * omega + R(15) * omega * omega);
    r.minusTau = -R(1) * (R(1) / omega - R(1) / R(2));
    r.halfMinusOmega = R(1) / R(2) * (-omega);
    r.omegaThreeHalves = omega * (R(3) / R(2));
    r.minusThreeOmega = -R(3) * omega;
    r.secondOrderCorrection = R(3) * (R(1) + R(1) / R(2) * (-omega));
    r.qlP = qlP;
    r.qlM = qlM;
    r.qlD = qlD;
    return r;
}

// ---------------------------------------------------------------- chimera --
// ChimeraTransformation.h:58-121 (Geier et al. 2015, appendix J)
template <class R>
__device__ __forceinline__ void fwdK(R& a, R& b, R& c, R vv, R v2, R kinv, R k)
{
    const R m2 = a + c;
    const R m1 = c - a;
    R m0 = m2 + b;
    a = m0;
    m0 *= kinv;
    m0 += R(1);
    b = (m1 * kinv - m0 * vv) * k;
    c = ((m2 - R(2) * m1 * vv) * kinv + v2 * m0) * k;
}

template <class R>
__device__ __forceinline__ void bwdK(R& a, R& b, R& c, R vv, R v2, R kinv, R k)
{
    const R m0 = (((c - b) * R(0.5) + b * vv) * kinv + (a * kinv + R(1)) * (v2 - vv) * R(0.5)) * k;
    const R m1 = (((a - c) - R(2) * b * vv) * kinv + (a * kinv + R(1)) * (-v2)) * k;
    c = (((c + b) * R(0.5) + b * vv) * kinv + (a * kinv + R(1)) * (v2 + vv) * R(0.5)) * k;
    a = m0;
    b = m1;
}

template <class R>
__device__ __forceinline__ void fwd0(R& a, R& b, R& c, R vv, R v2)
{
    const R m1 = (a + c) + b;
    const R m2 = c - a;
    c = (c + a) + (v2 * m1 - R(2) * vv * m2);
    b = m2 - vv * m1;
    a = m1;
}

template <class R>
__device__ __forceinline__ void bwd0(R& a, R& b, R& c, R vv, R v2)
{
    const R ma = (c + a * (v2 - vv)) * R(0.5) + b * (vv - R(0.5));
    const R mb = ((a - c) - a * v2) - R(2) * b * vv;
    c = (c + a * (v2 + vv)) * R(0.5) + b * (vv + R(0.5));
    b = mb;
    a = ma;
}

// --------------------------------------------------------- macroscopic sums --
// MacroscopicQuantities.h:55-127 (pyramid summation)
template <class R>
__device__ __forceinline__ R pyramidDensity(const R* f)
{
    const R t1 = ((f[dPPP] + f[dMMM]) + (f[dMPM] + f[dPMP])) + ((f[dMPP] + f[dPMM]) + (f[dMMP] + f[dPPM]));
    const R t2 = (((f[d0MP] + f[d0PM]) + (f[d0MM] + f[d0PP])) + ((f[dM0P] + f[dP0M]) + (f[dM0M] + f[dP0P]))) +
                 ((f[dMP0] + f[dPM0]) + (f[dMM0] + f[dPP0]));
    const R t3 = ((f[dM00] + f[dP00]) + (f[d0M0] + f[d0P0])) + (f[d00M] + f[d00P]);
    return ((t1 + t2) + f[d000]) + t3;
}
template <class R>
__device__ __forceinline__ R pyramidJx(const R* f)
{
    return ((((f[dPPP] - f[dMMM]) + (f[dPMP] - f[dMPM])) + ((f[dPMM] - f[dMPP]) + (f[dPPM] - f[dMMP]))) +
            (((f[dP0M] - f[dM0P]) + (f[dP0P] - f[dM0M])) + ((f[dPM0] - f[dMP0]) + (f[dPP0] - f[dMM0])))) +
           (f[dP00] - f[dM00]);
}
template <class R>
__device__ __forceinline__ R pyramidJy(const R* f)
{
    return ((((f[dPPP] - f[dMMM]) + (f[dMPM] - f[dPMP])) + ((f[dMPP] - f[dPMM]) + (f[dPPM] - f[dMMP]))) +
            (((f[d0PM] - f[d0MP]) + (f[d0PP] - f[d0MM])) + ((f[dMP0] - f[dPM0]) + (f[dPP0] - f[dMM0])))) +
           (f[d0P0] - f[d0M0]);
}
template <class R>
__device__ __forceinline__ R pyramidJz(const R* f)
{
    return ((((f[dPPP] - f[dMMM]) + (f[dPMP] - f[dMPM])) + ((f[dMPP] - f[dPMM]) + (f[dMMP] - f[dPPM]))) +
            (((f[d0MP] - f[d0PM]) + (f[d0PP] - f[d0MM])) + ((f[dM0P] - f[dP0M]) + (f[dP0P] - f[dM0M])))) +
           (f[d00P] - f[d00M]);
}

// ------------------------------------------------------------------- K17 --
// sixth-order correction term of K17CompressibleNavierStokes.h:320-330 / :489-500
template <class R>
__device__ __forceinline__ R c222Term(R m111, R m200, R m020, R m002, R m022, R m202, R m220, R m011, R m101, R m110,
                                      R m211, R m121, R m112, R m120, R m102, R m210, R m012, R m201, R m021,
                                      R oneOverRho, R drho)
{
    return (-R(4) * m111 * m111 - (m200 * m022 + m020 * m202 + m002 * m220) -
            R(4) * (m011 * m211 + m101 * m121 + m110 * m112) - R(2) * (m120 * m102 + m210 * m012 + m201 * m021)) *
               oneOverRho +
           (R(4) * (m101 * m101 * m020 + m011 * m011 * m200 + m110 * m110 * m002) + R(2) * (m200 * m020 * m002) +
            R(16) * m110 * m101 * m011) *
               oneOverRho * oneOverRho -
           R(1) / R(3) * (m022 + m202 + m220) * oneOverRho - R(1) / R(9) * (m200 + m020 + m002) * oneOverRho +
           (R(2) * (m101 * m101 + m011 * m011 + m110 * m110) + (m002 * m020 + m002 * m200 + m020 * m200) +
            R(1) / R(3) * (m002 + m020 + m200)) *
               oneOverRho * oneOverRho * (R(2) / R(3)) +
           R(1) / R(27) * ((drho * drho - drho) * oneOverRho * oneOverRho);
}

// One K17 collision on f[27] (pre-collision in, post-collision out).
// (fx, fy, fz) is half the acceleration already scaled by the level factor
// (RunCollision.cuh:111-113).  Returns drho and the force-shifted velocity.
template <class R>
__device__ __forceinline__ void k17Collide(R* f, const K17Rates<R>& r, R fx, R fy, R fz, R& drho_out, R& vx_out,
                                           R& vy_out, R& vz_out)
{
    const R drho = pyramidDensity(f);
    const R oneOverRho = R(1) / (drho + R(1));
    R vvx = pyramidJx(f) * oneOverRho;
    R vvy = pyramidJy(f) * oneOverRho;
    R vvz = pyramidJz(f) * oneOverRho;
    vvx += fx;
    vvy += fy;
    vvz += fz;
    const R vx2 = vvx * vvx, vy2 = vvy * vvy, vz2 = vvz * vvz;

    // forward chimera, z then y then x (:190-222)
    fwdK(f[dMMM], f[dMM0], f[dMMP], vvz, vz2, R(36), R(1) / R(36));
    fwdK(f[dM0M], f[dM00], f[dM0P], vvz, vz2, R(9), R(1) / R(9));
    fwdK(f[dMPM], f[dMP0], f[dMPP], vvz, vz2, R(36), R(1) / R(36));
    fwdK(f[d0MM], f[d0M0], f[d0MP], vvz, vz2, R(9), R(1) / R(9));
    fwdK(f[d00M], f[d000], f[d00P], vvz, vz2, R(9) / R(4), R(4) / R(9));
    fwdK(f[d0PM], f[d0P0], f[d0PP], vvz, vz2, R(9), R(1) / R(9));
    fwdK(f[dPMM], f[dPM0], f[dPMP], vvz, vz2, R(36), R(1) / R(36));
    fwdK(f[dP0M], f[dP00], f[dP0P], vvz, vz2, R(9), R(1) / R(9));
    fwdK(f[dPPM], f[dPP0], f[dPPP], vvz, vz2, R(36), R(1) / R(36));

    fwdK(f[dMMM], f[dM0M], f[dMPM], vvy, vy2, R(6), R(1) / R(6));
    fwd0(f[dMM0], f[dM00], f[dMP0], vvy, vy2);
    fwdK(f[dMMP], f[dM0P], f[dMPP], vvy, vy2, R(18), R(1) / R(18));
    fwdK(f[d0MM], f[d00M], f[d0PM], vvy, vy2, R(3) / R(2), R(2) / R(3));
    fwd0(f[d0M0], f[d000], f[d0P0], vvy, vy2);
    fwdK(f[d0MP], f[d00P], f[d0PP], vvy, vy2, R(9) / R(2), R(2) / R(9));
    fwdK(f[dPMM], f[dP0M], f[dPPM], vvy, vy2, R(6), R(1) / R(6));
    fwd0(f[dPM0], f[dP00], f[dPP0], vvy, vy2);
    fwdK(f[dPMP], f[dP0P], f[dPPP], vvy, vy2, R(18), R(1) / R(18));

    fwdK(f[dMMM], f[d0MM], f[dPMM], vvx, vx2, R(1), R(1));
    fwd0(f[dM0M], f[d00M], f[dP0M], vvx, vx2);
    fwdK(f[dMPM], f[d0PM], f[dPPM], vvx, vx2, R(3), R(1) / R(3));
    fwd0(f[dMM0], f[d0M0], f[dPM0], vvx, vx2);
    fwd0(f[dM00], f[d000], f[dP00], vvx, vx2);
    fwd0(f[dMP0], f[d0P0], f[dPP0], vvx, vx2);
    fwdK(f[dMMP], f[d0MP], f[dPMP], vvx, vx2, R(3), R(1) / R(3));
    fwd0(f[dM0P], f[d00P], f[dP0P], vvx, vx2);
    // Kinverse = 3 with K = 1/9, as the reference header has it (:222)
    fwdK(f[dMPP], f[d0PP], f[dPPP], vvx, vx2, R(3), R(1) / R(9));

    // moment names: m_abc is stored in the slot of direction (a-1, b-1, c-1)
    R& m000 = f[dMMM];
    R& m100 = f[d0MM];
    R& m200 = f[dPMM];
    R& m010 = f[dM0M];
    R& m110 = f[d00M];
    R& m210 = f[dP0M];
    R& m020 = f[dMPM];
    R& m120 = f[d0PM];
    R& m220 = f[dPPM];
    R& m001 = f[dMM0];
    R& m101 = f[d0M0];
    R& m201 = f[dPM0];
    R& m011 = f[dM00];
    R& m111 = f[d000];
    R& m211 = f[dP00];
    R& m021 = f[dMP0];
    R& m121 = f[d0P0];
    R& m221 = f[dPP0];
    R& m002 = f[dMMP];
    R& m102 = f[d0MP];
    R& m202 = f[dPMP];
    R& m012 = f[dM0P];
    R& m112 = f[d00P];
    R& m212 = f[dP0P];
    R& m022 = f[dMPP];
    R& m122 = f[d0PP];
    R& m222 = f[dPPP];

    // second and third order combinations (:329-346)
    R mxxPyyPzz = m200 + m020 + m002;
    R mxxMyy = m200 - m020;
    R mxxMzz = m200 - m002;
    R mxxyPyzz = m210 + m012;
    R mxxyMyzz = m210 - m012;
    R mxxzPyyz = m201 + m021;
    R mxxzMyyz = m201 - m021;
    R mxyyPxzz = m120 + m102;
    R mxyyMxzz = m120 - m102;

    // velocity gradients (:357-362), OxxPyyPzz = 1
    const R Dxy = r.minusThreeOmega * m110;
    const R Dxz = r.minusThreeOmega * m101;
    const R Dyz = r.minusThreeOmega * m011;
    const R dxux = r.halfMinusOmega * (mxxMyy + mxxMzz) + R(0.5) * (m000 - mxxPyyPzz);
    const R dyuy = dxux + r.omegaThreeHalves * mxxMyy;
    const R dzuz = dxux + r.omegaThreeHalves * mxxMzz;

    // second order relaxation with correction (:387-389)
    mxxPyyPzz += (m000 - mxxPyyPzz) - R(1.5) * (vx2 * dxux + vy2 * dyuy + vz2 * dzuz);
    mxxMyy += r.omega * (-mxxMyy) - r.secondOrderCorrection * (vx2 * dxux - vy2 * dyuy);
    mxxMzz += r.omega * (-mxxMzz) - r.secondOrderCorrection * (vx2 * dxux - vz2 * dzuz);
    m011 += r.omega * (-m011);
    m101 += r.omega * (-m101);
    m110 += r.omega * (-m110);

    // third order with quartic limiter (:404-417)
    R w;
    w = r.Oxyz + r.oneMinusOxyz * fabs(m111) / (fabs(m111) + r.qlD);
    m111 += w * (-m111);
    w = r.OxyyPxzz + r.oneMinusOxyyPxzz * fabs(mxxyPyzz) / (fabs(mxxyPyzz) + r.qlP);
    mxxyPyzz += w * (-mxxyPyzz);
    w = r.OxyyMxzz + r.oneMinusOxyyMxzz * fabs(mxxyMyzz) / (fabs(mxxyMyzz) + r.qlM);
    mxxyMyzz += w * (-mxxyMyzz);
    w = r.OxyyPxzz + r.oneMinusOxyyPxzz * fabs(mxxzPyyz) / (fabs(mxxzPyyz) + r.qlP);
    mxxzPyyz += w * (-mxxzPyyz);
    w = r.OxyyMxzz + r.oneMinusOxyyMxzz * fabs(mxxzMyyz) / (fabs(mxxzMyyz) + r.qlM);
    mxxzMyyz += w * (-mxxzMyyz);
    w = r.OxyyPxzz + r.oneMinusOxyyPxzz * fabs(mxyyPxzz) / (fabs(mxyyPxzz) + r.qlP);
    mxyyPxzz += w * (-mxyyPxzz);
    w = r.OxyyMxzz + r.oneMinusOxyyMxzz * fabs(mxyyMxzz) / (fabs(mxyyMxzz) + r.qlM);
    mxyyMxzz += w * (-mxyyMxzz);

    // back to single moments (:431-441)
    m200 = R(1) / R(3) * (mxxMyy + mxxMzz + mxxPyyPzz);
    m020 = R(1) / R(3) * (-R(2) * mxxMyy + mxxMzz + mxxPyyPzz);
    m002 = R(1) / R(3) * (mxxMyy - R(2) * mxxMzz + mxxPyyPzz);
    m210 = (mxxyMyzz + mxxyPyzz) * R(0.5);
    m012 = (-mxxyMyzz + mxxyPyzz) * R(0.5);
    m201 = (mxxzMyyz + mxxzPyyz) * R(0.5);
    m021 = (-mxxzMyyz + mxxzPyyz) * R(0.5);
    m120 = (mxyyMxzz + mxyyPxzz) * R(0.5);
    m102 = (-mxyyMxzz + mxyyPxzz) * R(0.5);

    // fourth order to the modified equilibrium (:452-457); orders 5 and 6
    // relax to zero (:463-471)
    const R cm022 = r.minusTau * (dyuy + dzuz) * (R(2) / R(3)) * r.factorA;
    const R cm202 = r.minusTau * (dxux + dzuz) * (R(2) / R(3)) * r.factorA;
    const R cm220 = r.minusTau * (dyuy + dxux) * (R(2) / R(3)) * r.factorA;
    const R cm112 = r.minusTau * Dxy * (R(1) / R(3)) * r.factorB;
    const R cm121 = r.minusTau * Dxz * (R(1) / R(3)) * r.factorB;
    const R cm211 = r.minusTau * Dyz * (R(1) / R(3)) * r.factorB;

    // cumulants back to central moments (:478-505)
    m211 = cm211 + R(1) / R(3) * ((R(3) * m200 + R(1)) * m011 + R(6) * m110 * m101) * oneOverRho;
    m121 = cm121 + R(1) / R(3) * ((R(3) * m020 + R(1)) * m101 + R(6) * m110 * m011) * oneOverRho;
    m112 = cm112 + R(1) / R(3) * ((R(3) * m002 + R(1)) * m110 + R(6) * m101 * m011) * oneOverRho;
    m220 = cm220 + (((m200 * m020 + R(2) * m110 * m110) * R(9) + R(3) * (m200 + m020)) * oneOverRho - (drho * oneOverRho)) *
                       (R(1) / R(9));
    m202 = cm202 + (((m200 * m002 + R(2) * m101 * m101) * R(9) + R(3) * (m200 + m002)) * oneOverRho - (drho * oneOverRho)) *
                       (R(1) / R(9));
    m022 = cm022 + (((m002 * m020 + R(2) * m011 * m011) * R(9) + R(3) * (m002 + m020)) * oneOverRho - (drho * oneOverRho)) *
                       (R(1) / R(9));
    m122 = R(1) / R(3) *
           (R(3) * (m002 * m120 + m020 * m102 + R(4) * m011 * m111 + R(2) * (m101 * m021 + m110 * m012)) + (m120 + m102)) *
           oneOverRho;
    m212 = R(1) / R(3) *
           (R(3) * (m002 * m210 + m200 * m012 + R(4) * m101 * m111 + R(2) * (m011 * m201 + m110 * m102)) + (m210 + m012)) *
           oneOverRho;
    m221 = R(1) / R(3) *
           (R(3) * (m200 * m021 + m020 * m201 + R(4) * m110 * m111 + R(2) * (m101 * m120 + m011 * m210)) + (m021 + m201)) *
           oneOverRho;
    m222 = -c222Term(m111, m200, m020, m002, m022, m202, m220, m011, m101, m110, m211, m121, m112, m120, m102, m210,
                     m012, m201, m021, oneOverRho, drho);

    // first moments change sign (force, :512-514)
    m100 = -m100;
    m010 = -m010;
    m001 = -m001;

    // backward chimera, x then y then z (:525-557)
    bwdK(m000, m100, m200, vvx, vx2, R(1), R(1));
    bwd0(m010, m110, m210, vvx, vx2);
    bwdK(m020, m120, m220, vvx, vx2, R(3), R(1) / R(3));
    bwd0(m001, m101, m201, vvx, vx2);
    bwd0(m011, m111, m211, vvx, vx2);
    bwd0(m021, m121, m221, vvx, vx2);
    bwdK(m002, m102, m202, vvx, vx2, R(3), R(1) / R(3));
    bwd0(m012, m112, m212, vvx, vx2);
    bwdK(m022, m122, m222, vvx, vx2, R(9), R(1) / R(9));

    bwdK(m000, m010, m020, vvy, vy2, R(6), R(1) / R(6));
    bwd0(m001, m011, m021, vvy, vy2);
    bwdK(m002, m012, m022, vvy, vy2, R(18), R(1) / R(18));
    bwdK(m100, m110, m120, vvy, vy2, R(3) / R(2), R(2) / R(3));
    bwd0(m101, m111, m121, vvy, vy2);
    bwdK(m102, m112, m122, vvy, vy2, R(9) / R(2), R(2) / R(9));
    bwdK(m200, m210, m220, vvy, vy2, R(6), R(1) / R(6));
    bwd0(m201, m211, m221, vvy, vy2);
    bwdK(m202, m212, m222, vvy, vy2, R(18), R(1) / R(18));

    bwdK(m000, m001, m002, vvz, vz2, R(36), R(1) / R(36));
    bwdK(m010, m011, m012, vvz, vz2, R(9), R(1) / R(9));
    bwdK(m020, m021, m022, vvz, vz2, R(36), R(1) / R(36));
    bwdK(m100, m101, m102, vvz, vz2, R(9), R(1) / R(9));
    bwdK(m110, m111, m112, vvz, vz2, R(9) / R(4), R(4) / R(9));
    bwdK(m120, m121, m122, vvz, vz2, R(9), R(1) / R(9));
    bwdK(m200, m201, m202, vvz, vz2, R(36), R(1) / R(36));
    bwdK(m210, m211, m212, vvz, vz2, R(9), R(1) / R(9));
    bwdK(m220, m221, m222, vvz, vz2, R(36), R(1) / R(36));

    drho_out = drho;
    vx_out = vvx;
    vy_out = vvy;
    vz_out = vvz;
}

// ------------------------------------------------------------------- BGK --
template <class R>
__device__ __forceinline__ void bgkCollide(R* f, R omega)
{
    R drho = (f[dPPP] + f[dMMM]) + (f[dMMP] + f[dPPM]) + (f[dPMP] + f[dMPM]) + (f[dMPP] + f[dPMM]) +
             (f[dPP0] + f[dMM0]) + (f[dMP0] + f[dPM0]) + (f[dP0P] + f[dM0M]) + (f[dP0M] + f[dM0P]) +
             (f[d0PP] + f[d0MM]) + (f[d0PM] + f[d0MP]) + (f[dP00] + f[dM00]) + (f[d0P0] + f[d0M0]) +
             (f[d00P] + f[d00M]) + f[d000];
    const R rho = drho + R(1);
    const R OORho = R(1) / rho;
    const R vx1 = OORho * ((f[dPPP] - f[dMMM]) + (f[dPPM] - f[dMMP]) + (f[dPMP] - f[dMPM]) + (f[dPMM] - f[dMPP]) +
                           (f[dPP0] - f[dMM0]) + (f[dPM0] - f[dMP0]) + (f[dP0P] - f[dM0M]) + (f[dP0M] - f[dM0P]) +
                           (f[dP00] - f[dM00]));
    const R vx2 = OORho * ((f[dPPP] - f[dMMM]) + (f[dPPM] - f[dMMP]) + (f[dMPM] - f[dPMP]) + (f[dMPP] - f[dPMM]) +
                           (f[dPP0] - f[dMM0]) + (f[dMP0] - f[dPM0]) + (f[d0PP] - f[d0MM]) + (f[d0PM] - f[d0MP]) +
                           (f[d0P0] - f[d0M0]));
    const R vx3 = OORho * ((f[dPPP] - f[dMMM]) + (f[dMMP] - f[dPPM]) + (f[dPMP] - f[dMPM]) + (f[dMPP] - f[dPMM]) +
                           (f[dP0P] - f[dM0M]) + (f[dM0P] - f[dP0M]) + (f[d0PP] - f[d0MM]) + (f[d0MP] - f[d0PM]) +
                           (f[d00P] - f[d00M]));
    const R cusq = R(1.5) * (vx1 * vx1 + vx2 * vx2 + vx3 * vx3);
    const R keep = R(1) + (-omega);
    f[d000] = f[d000] * keep - (-omega) * weight<R>(d000) * (drho - rho * cusq);
#pragma unroll
    for (int d = 1; d < 27; ++d) {
        const R cu = cdot<R>(d, vx1, vx2, vx3);
        f[d] = f[d] * keep - (-omega) * weight<R>(d) * (drho + rho * (R(3) * cu + R(4.5) * cu * cu - cusq));
    }
}

} // namespace vfb
