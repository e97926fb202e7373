// collision_math.cuh -- per-node collision operators, held in registers.
//
// K17: the compressible cumulant collision of VirtualFluids
// (src/lbm/collision/K17CompressibleNavierStokes.h:87-591, TurbulenceModel::None),
// based on Geier et al., J. Comput. Phys. 348 (2017) 862-888 and 889-898.
// The operator is the reference's, term for term; the arithmetic is arranged
// for the GPU's issue rate (the step is instruction bound at ~1 kflop/node):
//   * the chimera transforms are written in multiply-add form with their
//     conditioning factors multiplied out (algebraically identical);
//   * density, momentum and the first (z) chimera sweep share the sums over
//     the nine z lines of the lattice;
//   * rates that depend only on omega and the limiters are formed once per
//     launch on the host (K17Rates) with the reference's expressions;
//   * cumulants whose post-collision value does not depend on their
//     pre-collision value (orders 4..6 with O4 = O5 = O6 = 1) are never
//     formed: the reference computes them and then multiplies them by
//     (1 - 1) = 0 or cancels them exactly (x + 1 * (-x) = +0);
//   * in FP32 the seven limiter quotients use the fast division.
// Results agree with the reference to rounding: FP64 fields within 1e-12
// relative of the oracle after many steps (tests/test_gpu_collision.py).
//
// BGK: src/gpu/core/Kernel/Compressible/NavierStokes/B92/B92CompressibleNavierStokes_Device.cu:194-234.
#pragma once

#include "d3q27.cuh"

namespace vfb
{

// The scalar type behind an arithmetic type R (R itself for float / double;
// a paired type maps to its element type), and the rational constants of the
// operator as compile-time scalars converted to R.
template <class R>
struct ScalarOf {
    using type = R;
};
template <class R>
__host__ __device__ __forceinline__ R cst(int n, int m)
{
    using S = typename ScalarOf<R>::type;
    return R(S(n) / S(m));
}

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
    // per-launch factors of the fourth-order terms (:452-457):
    // minusTau * 2/3 * factorA, minusTau * (-3 omega) * 1/3 * factorB
    R fourthA, fourthB;
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
    r.minusTau = -R(1) * (R(1) / omega - cst<R>(1, 2));
    r.halfMinusOmega = cst<R>(1, 2) * (-omega);
    r.omegaThreeHalves = omega * (cst<R>(3, 2));
    r.minusThreeOmega = -R(3) * omega;
    r.secondOrderCorrection = R(3) * (R(1) + cst<R>(1, 2) * (-omega));
    r.qlP = qlP;
    r.qlM = qlM;
    r.qlD = qlD;
    r.fourthA = r.minusTau * cst<R>(2, 3) * r.factorA;
    r.fourthB = r.minusTau * r.minusThreeOmega * cst<R>(1, 3) * r.factorB;
    return r;
}

// ---------------------------------------------------------------- chimera --
// Central-moment transforms of ChimeraTransformation.h:58-121 (Geier et al.
// 2015, appendix J), written in multiply-add form.  With the conditioning pair
// (Kinverse, K) of a line and Kq = Kinverse * K:
//   forward   a' = a + b + c
//             b' = Kq (m1 - vv m0) - K vv,      m1 = c - a, m2 = a + c, m0 = a'
//             c' = Kq (m2 - 2 vv m1 + v2 m0) + K v2
//   backward  a' = c/2 + b (vv - 1/2) + (a + K) (v2 - vv)/2
//             b' = (a - c) - 2 vv b - v2 (a + K)
//             c' = c/2 + b (vv + 1/2) + (a + K) (v2 + vv)/2
// which are the reference's expressions with the factors Kinverse and K
// multiplied out (every line has Kq = 1 except the last forward x line, whose
// pair (3, 1/9) gives Kq = 1/3; K = 0 gives the plain transforms).
template <class R>
struct Sweep {
    R vv, v2, nvv, n2vv, nv2, hm, hp, vvm, vvp;
    __host__ __device__ __forceinline__ Sweep(R v)
    {
        vv = v;
        v2 = v * v;
        nvv = -v;
        n2vv = R(-2) * v;
        nv2 = -v2;
        hm = R(0.5) * (v2 - v);
        hp = R(0.5) * (v2 + v);
        vvm = v - R(0.5);
        vvp = v + R(0.5);
    }
};

template <class R>
__host__ __device__ __forceinline__ void fwd(R& a, R& b, R& c, const Sweep<R>& w, typename ScalarOf<R>::type K)
{
    const R m2 = a + c;
    const R m1 = c - a;
    const R m0 = m2 + b;
    const R m0K = K != 0 ? m0 + R(K) : m0;
    a = m0;
    b = fma(w.nvv, m0K, m1);
    c = fma(w.v2, m0K, fma(w.n2vv, m1, m2));
}

// the forward x line with (Kinverse, K) = (3, 1/9) of K17CompressibleNavierStokes.h:222
template <class R>
__host__ __device__ __forceinline__ void fwdThird(R& a, R& b, R& c, const Sweep<R>& w)
{
    const R m2 = a + c;
    const R m1 = c - a;
    const R m0 = m2 + b;
    a = m0;
    b = fma(cst<R>(1, 3), fma(w.nvv, m0, m1), w.nvv * (cst<R>(1, 9)));
    c = fma(cst<R>(1, 3), fma(w.v2, m0, fma(w.n2vv, m1, m2)), w.v2 * (cst<R>(1, 9)));
}

template <class R>
__host__ __device__ __forceinline__ void bwd(R& a, R& b, R& c, const Sweep<R>& w, typename ScalarOf<R>::type K)
{
    const R aK = K != 0 ? a + R(K) : a;
    const R hc = R(0.5) * c;
    const R na = fma(aK, w.hm, fma(b, w.vvm, hc));
    if constexpr (sizeof(typename ScalarOf<R>::type) == 8) {
        // FP64: three independent chains (measured faster in double precision)
        const R nb = fma(w.nv2, aK, fma(w.n2vv, b, a - c));
        c = fma(aK, w.hp, fma(b, w.vvp, hc));
        a = na;
        b = nb;
    } else {
        // FP32 (scalar or paired): two operations fewer; hp - hm = v and
        // vvp - vvm = 1, and the three populations sum to a
        const R nc = na + fma(aK, w.vv, b);
        b = (a - na) - nc;
        a = na;
        c = nc;
    }
}

// --------------------------------------------------------- macroscopic sums --
// MacroscopicQuantities.h:55-127 (pyramid summation)
template <class R>
__host__ __device__ __forceinline__ R pyramidDensity(const R* f)
{
    const R t1 = ((f[dPPP] + f[dMMM]) + (f[dMPM] + f[dPMP])) + ((f[dMPP] + f[dPMM]) + (f[dMMP] + f[dPPM]));
    const R t2 = (((f[d0MP] + f[d0PM]) + (f[d0MM] + f[d0PP])) + ((f[dM0P] + f[dP0M]) + (f[dM0M] + f[dP0P]))) +
                 ((f[dMP0] + f[dPM0]) + (f[dMM0] + f[dPP0]));
    const R t3 = ((f[dM00] + f[dP00]) + (f[d0M0] + f[d0P0])) + (f[d00M] + f[d00P]);
    return ((t1 + t2) + f[d000]) + t3;
}
template <class R>
__host__ __device__ __forceinline__ R pyramidJx(const R* f)
{
    return ((((f[dPPP] - f[dMMM]) + (f[dPMP] - f[dMPM])) + ((f[dPMM] - f[dMPP]) + (f[dPPM] - f[dMMP]))) +
            (((f[dP0M] - f[dM0P]) + (f[dP0P] - f[dM0M])) + ((f[dPM0] - f[dMP0]) + (f[dPP0] - f[dMM0])))) +
           (f[dP00] - f[dM00]);
}
template <class R>
__host__ __device__ __forceinline__ R pyramidJy(const R* f)
{
    return ((((f[dPPP] - f[dMMM]) + (f[dMPM] - f[dPMP])) + ((f[dMPP] - f[dPMM]) + (f[dPPM] - f[dMMP]))) +
            (((f[d0PM] - f[d0MP]) + (f[d0PP] - f[d0MM])) + ((f[dMP0] - f[dPM0]) + (f[dPP0] - f[dMM0])))) +
           (f[d0P0] - f[d0M0]);
}
template <class R>
__host__ __device__ __forceinline__ R pyramidJz(const R* f)
{
    return ((((f[dPPP] - f[dMMM]) + (f[dPMP] - f[dMPM])) + ((f[dMPP] - f[dPMM]) + (f[dMMP] - f[dPPM]))) +
            (((f[d0MP] - f[d0PM]) + (f[d0PP] - f[d0MM])) + ((f[dM0P] - f[dP0M]) + (f[dP0P] - f[dM0M])))) +
           (f[d00P] - f[d00M]);
}

// ------------------------------------------------------------------- K17 --
// sixth-order correction term of K17CompressibleNavierStokes.h:320-330 / :489-500,
// regrouped as (A + B / rho) / rho: A collects the terms over rho, B those
// over rho^2 (the same terms, fused multiply-adds)
template <class R>
__host__ __device__ __forceinline__ R c222Term(R m111, R m200, R m020, R m002, R m022, R m202, R m220, R m011, R m101, R m110,
                                      R m211, R m121, R m112, R m120, R m102, R m210, R m012, R m201, R m021,
                                      R oneOverRho, R drho)
{
    const R s2 = m200 + m020 + m002;
    const R a1 = fma(m002, m220, fma(m020, m202, m200 * m022));
    const R a2 = fma(m110, m112, fma(m101, m121, m011 * m211));
    const R a3 = fma(m201, m021, fma(m210, m012, m120 * m102));
    R A = fma(R(-4), m111 * m111, -a1);
    A = fma(R(-4), a2, A);
    A = fma(R(-2), a3, A);
    A = fma(-cst<R>(1, 3), m022 + m202 + m220, A);
    A = fma(-cst<R>(1, 9), s2, A);
    const R q101 = m101 * m101, q011 = m011 * m011, q110 = m110 * m110;
    const R m200m020 = m200 * m020;
    const R b1 = fma(q110, m002, fma(q011, m200, q101 * m020));
    const R pairs = fma(m002, m020, fma(m002, m200, m200m020));
    const R inner = fma(cst<R>(1, 3), s2, fma(R(2), q101 + q011 + q110, pairs));
    R B = fma(R(2), m200m020 * m002, R(4) * b1);
    B = fma(R(16), (m110 * m101) * m011, B);
    B = fma(cst<R>(2, 3), inner, B);
    B = fma(cst<R>(1, 27), fma(drho, drho, -drho), B);
    return fma(B, oneOverRho, A) * oneOverRho;
}

template <class R>
__host__ __device__ __forceinline__ R limiterQuotient(R x, R y)
{
    return x / y;
}
#ifdef __CUDA_ARCH__
template <>
__device__ __forceinline__ float limiterQuotient<float>(float x, float y)
{
    return __fdividef(x, y);
}
#endif

// Central moments (in the slots of k17Collide's naming: m_abc in the slot of
// direction (a-1, b-1, c-1)) to populations: the backward chimera transform
// in x, then y, then z (K17CompressibleNavierStokes.h:525-557; the same
// sequence closes the interface interpolation, InterpolationCF.h:250-285).
template <class R>
__host__ __device__ __forceinline__ void centralMomentsToPopulations(R* f, R vvx, R vvy, R vvz)
{
    {
        const Sweep<R> w(vvx);
        bwd(f[dMMM], f[d0MM], f[dPMM], w, typename ScalarOf<R>::type(1));
        bwd(f[dM0M], f[d00M], f[dP0M], w, typename ScalarOf<R>::type(0));
        bwd(f[dMPM], f[d0PM], f[dPPM], w, cst<typename ScalarOf<R>::type>(1, 3));
        bwd(f[dMM0], f[d0M0], f[dPM0], w, typename ScalarOf<R>::type(0));
        bwd(f[dM00], f[d000], f[dP00], w, typename ScalarOf<R>::type(0));
        bwd(f[dMP0], f[d0P0], f[dPP0], w, typename ScalarOf<R>::type(0));
        bwd(f[dMMP], f[d0MP], f[dPMP], w, cst<typename ScalarOf<R>::type>(1, 3));
        bwd(f[dM0P], f[d00P], f[dP0P], w, typename ScalarOf<R>::type(0));
        bwd(f[dMPP], f[d0PP], f[dPPP], w, cst<typename ScalarOf<R>::type>(1, 9));
    }
    {
        const Sweep<R> w(vvy);
        bwd(f[dMMM], f[dM0M], f[dMPM], w, cst<typename ScalarOf<R>::type>(1, 6));
        bwd(f[dMM0], f[dM00], f[dMP0], w, typename ScalarOf<R>::type(0));
        bwd(f[dMMP], f[dM0P], f[dMPP], w, cst<typename ScalarOf<R>::type>(1, 18));
        bwd(f[d0MM], f[d00M], f[d0PM], w, cst<typename ScalarOf<R>::type>(2, 3));
        bwd(f[d0M0], f[d000], f[d0P0], w, typename ScalarOf<R>::type(0));
        bwd(f[d0MP], f[d00P], f[d0PP], w, cst<typename ScalarOf<R>::type>(2, 9));
        bwd(f[dPMM], f[dP0M], f[dPPM], w, cst<typename ScalarOf<R>::type>(1, 6));
        bwd(f[dPM0], f[dP00], f[dPP0], w, typename ScalarOf<R>::type(0));
        bwd(f[dPMP], f[dP0P], f[dPPP], w, cst<typename ScalarOf<R>::type>(1, 18));
    }
    {
        const Sweep<R> w(vvz);
        bwd(f[dMMM], f[dMM0], f[dMMP], w, cst<typename ScalarOf<R>::type>(1, 36));
        bwd(f[dM0M], f[dM00], f[dM0P], w, cst<typename ScalarOf<R>::type>(1, 9));
        bwd(f[dMPM], f[dMP0], f[dMPP], w, cst<typename ScalarOf<R>::type>(1, 36));
        bwd(f[d0MM], f[d0M0], f[d0MP], w, cst<typename ScalarOf<R>::type>(1, 9));
        bwd(f[d00M], f[d000], f[d00P], w, cst<typename ScalarOf<R>::type>(4, 9));
        bwd(f[d0PM], f[d0P0], f[d0PP], w, cst<typename ScalarOf<R>::type>(1, 9));
        bwd(f[dPMM], f[dPM0], f[dPMP], w, cst<typename ScalarOf<R>::type>(1, 36));
        bwd(f[dP0M], f[dP00], f[dP0P], w, cst<typename ScalarOf<R>::type>(1, 9));
        bwd(f[dPPM], f[dPP0], f[dPPP], w, cst<typename ScalarOf<R>::type>(1, 36));
    }
}

// One K17 collision on f[27] (pre-collision in, post-collision out).
// (fx, fy, fz) is half the acceleration already scaled by the level factor
// (RunCollision.cuh:111-113).  Returns drho and the force-shifted velocity.
template <class R>
__host__ __device__ __forceinline__ void k17Collide(R* f, const K17Rates<R>& r, R fx, R fy, R fz, R& drho_out,
                                                    R& vx_out, R& vy_out, R& vz_out)
{
    // sums over the nine z lines (x, y fixed): s = a + b + c, m2 = a + c, d = c - a
#define VFB_ZLINE(XY, A, B, C)                                                                                         \
    const R m2_##XY = f[A] + f[C];                                                                                     \
    const R d_##XY = f[C] - f[A];                                                                                      \
    const R s_##XY = m2_##XY + f[B];
    VFB_ZLINE(MM, dMMM, dMM0, dMMP)
    VFB_ZLINE(M0, dM0M, dM00, dM0P)
    VFB_ZLINE(MP, dMPM, dMP0, dMPP)
    VFB_ZLINE(0M, d0MM, d0M0, d0MP)
    VFB_ZLINE(00, d00M, d000, d00P)
    VFB_ZLINE(0P, d0PM, d0P0, d0PP)
    VFB_ZLINE(PM, dPMM, dPM0, dPMP)
    VFB_ZLINE(P0, dP0M, dP00, dP0P)
    VFB_ZLINE(PP, dPPM, dPP0, dPPP)
#undef VFB_ZLINE
    const R drho = (((s_MM + s_PP) + (s_MP + s_PM)) + ((s_M0 + s_P0) + (s_0M + s_0P))) + s_00;
    const R jx = ((s_PM + s_PP) - (s_MM + s_MP)) + (s_P0 - s_M0);
    const R jy = ((s_MP + s_PP) - (s_MM + s_PM)) + (s_0P - s_0M);
    const R jz = (((d_MM + d_PP) + (d_MP + d_PM)) + ((d_M0 + d_P0) + (d_0M + d_0P))) + d_00;
    const R oneOverRho = R(1) / (drho + R(1));
    const R vvx = fma(jx, oneOverRho, fx);
    const R vvy = fma(jy, oneOverRho, fy);
    const R vvz = fma(jz, oneOverRho, fz);
    const R vx2 = vvx * vvx, vy2 = vvy * vvy, vz2 = vvz * vvz;

    // forward chimera in z (:190-199) from the line sums
    {
        const Sweep<R> w(vvz);
#define VFB_ZFWD(XY, A, B, C, K)                                                                                       \
    {                                                                                                                  \
        const R m0K = s_##XY + (K);                                                                                    \
        f[A] = s_##XY;                                                                                                 \
        f[B] = fma(w.nvv, m0K, d_##XY);                                                                                \
        f[C] = fma(w.v2, m0K, fma(w.n2vv, d_##XY, m2_##XY));                                                           \
    }
        VFB_ZFWD(MM, dMMM, dMM0, dMMP, cst<R>(1, 36))
        VFB_ZFWD(M0, dM0M, dM00, dM0P, cst<R>(1, 9))
        VFB_ZFWD(MP, dMPM, dMP0, dMPP, cst<R>(1, 36))
        VFB_ZFWD(0M, d0MM, d0M0, d0MP, cst<R>(1, 9))
        VFB_ZFWD(00, d00M, d000, d00P, cst<R>(4, 9))
        VFB_ZFWD(0P, d0PM, d0P0, d0PP, cst<R>(1, 9))
        VFB_ZFWD(PM, dPMM, dPM0, dPMP, cst<R>(1, 36))
        VFB_ZFWD(P0, dP0M, dP00, dP0P, cst<R>(1, 9))
        VFB_ZFWD(PP, dPPM, dPP0, dPPP, cst<R>(1, 36))
#undef VFB_ZFWD
    }
    // y (:202-210)
    {
        const Sweep<R> w(vvy);
        fwd(f[dMMM], f[dM0M], f[dMPM], w, cst<typename ScalarOf<R>::type>(1, 6));
        fwd(f[dMM0], f[dM00], f[dMP0], w, typename ScalarOf<R>::type(0));
        fwd(f[dMMP], f[dM0P], f[dMPP], w, cst<typename ScalarOf<R>::type>(1, 18));
        fwd(f[d0MM], f[d00M], f[d0PM], w, cst<typename ScalarOf<R>::type>(2, 3));
        fwd(f[d0M0], f[d000], f[d0P0], w, typename ScalarOf<R>::type(0));
        fwd(f[d0MP], f[d00P], f[d0PP], w, cst<typename ScalarOf<R>::type>(2, 9));
        fwd(f[dPMM], f[dP0M], f[dPPM], w, cst<typename ScalarOf<R>::type>(1, 6));
        fwd(f[dPM0], f[dP00], f[dPP0], w, typename ScalarOf<R>::type(0));
        fwd(f[dPMP], f[dP0P], f[dPPP], w, cst<typename ScalarOf<R>::type>(1, 18));
    }
    // x (:213-222)
    {
        const Sweep<R> w(vvx);
        fwd(f[dMMM], f[d0MM], f[dPMM], w, typename ScalarOf<R>::type(1));
        fwd(f[dM0M], f[d00M], f[dP0M], w, typename ScalarOf<R>::type(0));
        fwd(f[dMPM], f[d0PM], f[dPPM], w, cst<typename ScalarOf<R>::type>(1, 3));
        fwd(f[dMM0], f[d0M0], f[dPM0], w, typename ScalarOf<R>::type(0));
        fwd(f[dM00], f[d000], f[dP00], w, typename ScalarOf<R>::type(0));
        fwd(f[dMP0], f[d0P0], f[dPP0], w, typename ScalarOf<R>::type(0));
        fwd(f[dMMP], f[d0MP], f[dPMP], w, cst<typename ScalarOf<R>::type>(1, 3));
        fwd(f[dM0P], f[d00P], f[dP0P], w, typename ScalarOf<R>::type(0));
        fwdThird(f[dMPP], f[d0PP], f[dPPP], w);
    }

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

    // velocity gradients (:357-362), OxxPyyPzz = 1; the mixed ones (from the
    // second-order moments before relaxation) enter only the fourth-order
    // terms, through fourthB
    const R cm112 = r.fourthB * m110;
    const R cm121 = r.fourthB * m101;
    const R cm211 = r.fourthB * m011;
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
    w = fma(r.oneMinusOxyz, limiterQuotient(fabs(m111), fabs(m111) + r.qlD), r.Oxyz);
    m111 += w * (-m111);
    w = fma(r.oneMinusOxyyPxzz, limiterQuotient(fabs(mxxyPyzz), fabs(mxxyPyzz) + r.qlP), r.OxyyPxzz);
    mxxyPyzz += w * (-mxxyPyzz);
    w = fma(r.oneMinusOxyyMxzz, limiterQuotient(fabs(mxxyMyzz), fabs(mxxyMyzz) + r.qlM), r.OxyyMxzz);
    mxxyMyzz += w * (-mxxyMyzz);
    w = fma(r.oneMinusOxyyPxzz, limiterQuotient(fabs(mxxzPyyz), fabs(mxxzPyyz) + r.qlP), r.OxyyPxzz);
    mxxzPyyz += w * (-mxxzPyyz);
    w = fma(r.oneMinusOxyyMxzz, limiterQuotient(fabs(mxxzMyyz), fabs(mxxzMyyz) + r.qlM), r.OxyyMxzz);
    mxxzMyyz += w * (-mxxzMyyz);
    w = fma(r.oneMinusOxyyPxzz, limiterQuotient(fabs(mxyyPxzz), fabs(mxyyPxzz) + r.qlP), r.OxyyPxzz);
    mxyyPxzz += w * (-mxyyPxzz);
    w = fma(r.oneMinusOxyyMxzz, limiterQuotient(fabs(mxyyMxzz), fabs(mxyyMxzz) + r.qlM), r.OxyyMxzz);
    mxyyMxzz += w * (-mxyyMxzz);

    // back to single moments (:431-441)
    // (1/3)(-2 a + b + c) = (1/3)(a + b + c) - a, likewise for m002
    m200 = cst<R>(1, 3) * (mxxMyy + mxxMzz + mxxPyyPzz);
    m020 = m200 - mxxMyy;
    m002 = m200 - mxxMzz;
    m210 = (mxxyMyzz + mxxyPyzz) * R(0.5);
    m012 = (-mxxyMyzz + mxxyPyzz) * R(0.5);
    m201 = (mxxzMyyz + mxxzPyyz) * R(0.5);
    m021 = (-mxxzMyyz + mxxzPyyz) * R(0.5);
    m120 = (mxyyMxzz + mxyyPxzz) * R(0.5);
    m102 = (-mxyyMxzz + mxyyPxzz) * R(0.5);

    // fourth order to the modified equilibrium (:452-457); orders 5 and 6
    // relax to zero (:463-471)
    const R cm022 = r.fourthA * (dyuy + dzuz);
    const R cm202 = r.fourthA * (dxux + dzuz);
    const R cm220 = r.fourthA * (dyuy + dxux);

    // cumulants back to central moments (:478-505)
    // (the reference's (1/3) X / rho and (9 P + 3 S) / (9 rho) - drho / (9 rho)
    // regrouped as X (1/(3 rho)) and P / rho + S / (3 rho) - drho / (9 rho))
    const R oor3 = oneOverRho * cst<R>(1, 3);
    const R dr9 = drho * oneOverRho * cst<R>(1, 9);
    m211 = fma(fma(fma(R(3), m200, R(1)), m011, R(6) * (m110 * m101)), oor3, cm211);
    m121 = fma(fma(fma(R(3), m020, R(1)), m101, R(6) * (m110 * m011)), oor3, cm121);
    m112 = fma(fma(fma(R(3), m002, R(1)), m110, R(6) * (m101 * m011)), oor3, cm112);
    m220 = fma(fma(m200, m020, R(2) * (m110 * m110)), oneOverRho, fma(m200 + m020, oor3, cm220 - dr9));
    m202 = fma(fma(m200, m002, R(2) * (m101 * m101)), oneOverRho, fma(m200 + m002, oor3, cm202 - dr9));
    m022 = fma(fma(m002, m020, R(2) * (m011 * m011)), oneOverRho, fma(m002 + m020, oor3, cm022 - dr9));
    m122 = fma(fma(m002, m120, fma(m020, m102, fma(R(4) * m011, m111, R(2) * fma(m101, m021, m110 * m012)))),
               oneOverRho, (m120 + m102) * oor3);
    m212 = fma(fma(m002, m210, fma(m200, m012, fma(R(4) * m101, m111, R(2) * fma(m011, m201, m110 * m102)))),
               oneOverRho, (m210 + m012) * oor3);
    m221 = fma(fma(m200, m021, fma(m020, m201, fma(R(4) * m110, m111, R(2) * fma(m101, m120, m011 * m210)))),
               oneOverRho, (m021 + m201) * oor3);
    m222 = -c222Term(m111, m200, m020, m002, m022, m202, m220, m011, m101, m110, m211, m121, m112, m120, m102, m210,
                     m012, m201, m021, oneOverRho, drho);

    // first moments change sign (force, :512-514)
    m100 = -m100;
    m010 = -m010;
    m001 = -m001;

    // backward chimera, x then y then z (:525-557)
    centralMomentsToPopulations(f, vvx, vvy, vvz);

    drho_out = drho;
    vx_out = vvx;
    vy_out = vvy;
    vz_out = vvz;
}

// ------------------------------------------------------------------- BGK --
template <class R>
__host__ __device__ __forceinline__ void bgkCollide(R* f, R omega)
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
    // the weights as compile-time scalars (for a paired type R this avoids a
    // runtime division per direction; for float / double it is weight<R>)
    using S = typename ScalarOf<R>::type;
    f[d000] = f[d000] * keep - (-omega) * R(weight<S>(d000)) * (drho - rho * cusq);
#pragma unroll
    for (int d = 1; d < 27; ++d) {
        const R cu = cdot<R>(d, vx1, vx2, vx3);
        f[d] = f[d] * keep - (-omega) * R(weight<S>(d)) * (drho + rho * (R(3) * cu + R(4.5) * cu * cu - cusq));
    }
}

} // namespace vfb
