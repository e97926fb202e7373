// interpolation.cuh -- compressible coarse/fine interpolation of the
// refinement interface (host and device).
//
// The operator of VirtualFluids' scaleCoarseToFineCompressible /
// scaleFineToCoarseCompressible (src/lbm/interpolation/InterpolationCoefficients.h:86-430,
// src/lbm/refinement/InterpolationCF.h:57-306, InterpolationFC.h:56-263):
//  1. on each of the 8 source nodes of a cell: drho and velocity (pyramid
//     sums) and the five non-equilibrium second moments scaled by -3 omega
//     (xy, yz, xz) or -3/2 omega (xx-yy, xx-zz);
//  2. the coefficients of a polynomial that is quadratic in space (with the
//     tri-linear terms), fitted to the corner values and slopes, shifted by
//     the cell's offset vector for refinement into a wall;
//  3. on each destination node: drho, velocity and second-order
//     non-equilibrium moments from the polynomial, third order zero, fourth
//     order drho / 9, sixth drho / 27, and the backward chimera transform.
//
// Every coefficient is a signed sum over the corners, sum_c s(c) q(c), where
// s is a product of the corner's axis signs.  Here all eight such sums of a
// corner quantity come from one three-stage butterfly (a Walsh-Hadamard
// transform over the corner index), and the coefficients are formed from
// them.  The result equals the reference's to rounding.
#pragma once

#include "collision_math.cuh"
#include "d3q27.cuh"

namespace vfb
{

// the interpolation polynomial (names as the reference's coefficients)
template <class R>
struct InterpCoeffs {
    R a000, a100, a010, a001, a200, a020, a002, a110, a101, a011, a111;
    R b000, b100, b010, b001, b200, b020, b002, b110, b101, b011, b111;
    R c000, c100, c010, c001, c200, c020, c002, c110, c101, c011, c111;
    R d000, d100, d010, d001, d110, d101, d011, d111;
    R LaplaceRho;
};

// the nine quantities of one source node
template <class R>
struct SourceMoments {
    R drho, vx, vy, vz, kxy, kyz, kxz, kxxMyy, kxxMzz;
};

// MomentsOnSourceNode::calculate (InterpolationCoefficients.h:86-144)
template <class R>
__host__ __device__ __forceinline__ SourceMoments<R> sourceMoments(const R* f, R omega)
{
    SourceMoments<R> m;
    m.drho = pyramidDensity(f);
    const R oneOverRho = R(1) / (m.drho + R(1));
    m.vx = pyramidJx(f) * oneOverRho;
    m.vy = pyramidJy(f) * oneOverRho;
    m.vz = pyramidJz(f) * oneOverRho;
    // second moments sum_d c_a c_b f_d over the directions that carry them
    const R sxy = ((f[dPP0] + f[dMM0]) - (f[dPM0] + f[dMP0])) + ((f[dPPP] + f[dMMM]) + (f[dPPM] + f[dMMP])) -
                  ((f[dPMP] + f[dMPM]) + (f[dPMM] + f[dMPP]));
    const R syz = ((f[d0PP] + f[d0MM]) - (f[d0PM] + f[d0MP])) + ((f[dPPP] + f[dMMM]) + (f[dMPP] + f[dPMM])) -
                  ((f[dPPM] + f[dMMP]) + (f[dMPM] + f[dPMP]));
    const R sxz = ((f[dP0P] + f[dM0M]) - (f[dP0M] + f[dM0P])) + ((f[dPPP] + f[dMMM]) + (f[dPMP] + f[dMPM])) -
                  ((f[dPPM] + f[dMMP]) + (f[dPMM] + f[dMPP]));
    // xx - yy: directions with an x and no y component minus those with a y and no x component
    const R xOnly = (f[dP00] + f[dM00]) + ((f[dP0P] + f[dM0M]) + (f[dP0M] + f[dM0P]));
    const R yOnly = (f[d0P0] + f[d0M0]) + ((f[d0PP] + f[d0MM]) + (f[d0PM] + f[d0MP]));
    const R xNoZ = (f[dP00] + f[dM00]) + ((f[dPP0] + f[dMM0]) + (f[dPM0] + f[dMP0]));
    const R zNoX = (f[d00P] + f[d00M]) + ((f[d0PP] + f[d0MM]) + (f[d0PM] + f[d0MP]));
    m.kxy = -R(3) * omega * (sxy * oneOverRho - m.vx * m.vy);
    m.kyz = -R(3) * omega * (syz * oneOverRho - m.vy * m.vz);
    m.kxz = -R(3) * omega * (sxz * oneOverRho - m.vx * m.vz);
    m.kxxMyy = -R(3) / R(2) * omega * ((xOnly - yOnly) * oneOverRho - (m.vx * m.vx - m.vy * m.vy));
    m.kxxMzz = -R(3) / R(2) * omega * ((xNoZ - zNoX) * oneOverRho - (m.vx * m.vx - m.vz * m.vz));
    return m;
}

// signed corner sums of q over corners c = x | y << 1 | z << 2 (bit set: the
// positive side): out[m] = sum_c q[c] * prod over the axes in m of (+1 or -1)
template <class R>
__host__ __device__ __forceinline__ void cornerSums(const R* q, R* out)
{
    R t[8];
#pragma unroll
    for (int c = 0; c < 8; ++c)
        t[c] = q[c];
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        const int bit = 1 << axis;
#pragma unroll
        for (int c = 0; c < 8; ++c)
            if (!(c & bit)) {
                const R minus = t[c], plus = t[c | bit];
                t[c] = plus + minus;       // axis not in m
                t[c | bit] = plus - minus; // axis in m
            }
    }
#pragma unroll
    for (int m = 0; m < 8; ++m)
        out[m] = t[m];
}

// index of a sum in cornerSums' output
enum CornerSum : int { S1 = 0, SX = 1, SY = 2, SXY = 3, SZ = 4, SXZ = 5, SYZ = 6, SXYZ = 7 };

// MomentsOnSourceNodeSet::calculateCoefficients (InterpolationCoefficients.h:201-430)
template <class R>
__host__ __device__ __forceinline__ InterpCoeffs<R> interpolationCoefficients(const SourceMoments<R>* src, R xoff,
                                                                              R yoff, R zoff)
{
    R q[8], vx[8], vy[8], vz[8], dr[8], kxy[8], kyz[8], kxz[8], kmy[8], kmz[8];
#define VFB_CORNERS(OUT, FIELD)                                                                                        \
    _Pragma("unroll") for (int c = 0; c < 8; ++c) q[c] = src[c].FIELD;                                                 \
    cornerSums(q, OUT);
    VFB_CORNERS(vx, vx)
    VFB_CORNERS(vy, vy)
    VFB_CORNERS(vz, vz)
    VFB_CORNERS(dr, drho)
    VFB_CORNERS(kxy, kxy)
    VFB_CORNERS(kyz, kyz)
    VFB_CORNERS(kxz, kxz)
    VFB_CORNERS(kmy, kxxMyy)
    VFB_CORNERS(kmz, kxxMzz)
#undef VFB_CORNERS
    InterpCoeffs<R> k;
    k.a000 = (R(2) * (((vy[SXY] + vz[SXZ]) - kxy[SY]) - kxz[SZ]) + R(8) * vx[S1] - (kmy[SX] + kmz[SX])) / R(64);
    k.b000 = (R(2) * (((kmy[SY] + vx[SXY]) + vz[SYZ]) - (kxy[SX] + kyz[SZ])) + R(8) * vy[S1] - kmz[SY]) / R(64);
    k.c000 = (R(2) * (((kmz[SZ] + vx[SXZ]) + vy[SYZ]) - (kxz[SX] + kyz[SY])) + R(8) * vz[S1] - kmy[SZ]) / R(64);
    k.a100 = vx[SX] / R(4);
    k.b100 = vy[SX] / R(4);
    k.c100 = vz[SX] / R(4);
    k.a010 = vx[SY] / R(4);
    k.b010 = vy[SY] / R(4);
    k.c010 = vz[SY] / R(4);
    k.a001 = vx[SZ] / R(4);
    k.b001 = vy[SZ] / R(4);
    k.c001 = vz[SZ] / R(4);
    k.a200 = (R(2) * (vy[SXY] + vz[SXZ]) + (kmy[SX] + kmz[SX])) / R(16);
    k.b200 = (kxy[SX] - R(2) * vx[SXY]) / R(8);
    k.c200 = (kxz[SX] - R(2) * vx[SXZ]) / R(8);
    k.a020 = (kxy[SY] - R(2) * vy[SXY]) / R(8);
    k.b020 = (R(2) * ((vx[SXY] + vz[SYZ]) - kmy[SY]) + kmz[SY]) / R(16);
    k.c020 = (kyz[SY] - R(2) * vy[SYZ]) / R(8);
    k.a002 = (kxz[SZ] - R(2) * vz[SXZ]) / R(8);
    k.b002 = (kyz[SZ] - R(2) * vz[SYZ]) / R(8);
    k.c002 = (R(2) * ((vx[SXZ] + vy[SYZ]) - kmz[SZ]) + kmy[SZ]) / R(16);
    k.a110 = vx[SXY] / R(2);
    k.b110 = vy[SXY] / R(2);
    k.c110 = vz[SXY] / R(2);
    k.a101 = vx[SXZ] / R(2);
    k.b101 = vy[SXZ] / R(2);
    k.c101 = vz[SXZ] / R(2);
    k.a011 = vx[SYZ] / R(2);
    k.b011 = vy[SYZ] / R(2);
    k.c011 = vz[SYZ] / R(2);
    k.a111 = vx[SXYZ];
    k.b111 = vy[SXYZ];
    k.c111 = vz[SXYZ];
    k.d000 = dr[S1] / R(8);
    k.d100 = dr[SX] / R(4);
    k.d010 = dr[SY] / R(4);
    k.d001 = dr[SZ] / R(4);
    k.d110 = dr[SXY] / R(2);
    k.d101 = dr[SXZ] / R(2);
    k.d011 = dr[SYZ] / R(2);
    k.d111 = dr[SXYZ];
    // the pressure Laplacian is only used without an offset (:383-385)
    k.LaplaceRho = (xoff != R(0) || yoff != R(0) || zoff != R(0))
                       ? R(0)
                       : -R(3) * (k.a100 * k.a100 + k.b010 * k.b010 + k.c001 * k.c001) -
                             R(6) * (k.b100 * k.a010 + k.c100 * k.a001 + k.c010 * k.b001);
    // shift to the offset point for refinement into a wall (:404-428)
    const R xx = xoff * xoff, yy = yoff * yoff, zz = zoff * zoff;
    const R xy = xoff * yoff, xz = xoff * zoff, yz = yoff * zoff;
#define VFB_SHIFT(P)                                                                                                   \
    k.P##000 = k.P##000 + xoff * k.P##100 + yoff * k.P##010 + zoff * k.P##001 + xx * k.P##200 + yy * k.P##020 +       \
               zz * k.P##002 + xy * k.P##110 + xz * k.P##101 + yz * k.P##011;                                          \
    k.P##100 = k.P##100 + R(2) * xoff * k.P##200 + yoff * k.P##110 + zoff * k.P##101;                                 \
    k.P##010 = k.P##010 + R(2) * yoff * k.P##020 + xoff * k.P##110 + zoff * k.P##011;                                 \
    k.P##001 = k.P##001 + R(2) * zoff * k.P##002 + xoff * k.P##101 + yoff * k.P##011;
    VFB_SHIFT(a)
    VFB_SHIFT(b)
    VFB_SHIFT(c)
#undef VFB_SHIFT
    k.d000 = k.d000 + xoff * k.d100 + yoff * k.d010 + zoff * k.d001 + xy * k.d110 + xz * k.d101 + yz * k.d011;
    k.d100 = k.d100 + yoff * k.d110 + zoff * k.d101;
    k.d010 = k.d010 + xoff * k.d110 + zoff * k.d011;
    k.d001 = k.d001 + xoff * k.d101 + yoff * k.d011;
    return k;
}

// Populations of a destination node from drho, velocity and the five
// second-order non-equilibrium moments: third order zero, fourth order
// drho / 9, sixth drho / 27, then the backward chimera transform (the moment
// slots are those of k17Collide).  (InterpolationCF.h:160-306, InterpolationFC.h:140-263)
template <class R>
__host__ __device__ __forceinline__ void populationsFromMoments(R* f, R press, R vvx, R vvy, R vvz, R mxxMyy,
                                                               R mxxMzz, R m011, R m101, R m110)
{
#pragma unroll
    for (int d = 0; d < 27; ++d)
        f[d] = R(0);
    f[dMMM] = press;                                         // m000
    f[dPMM] = R(1) / R(3) * (mxxMyy + mxxMzz + press);       // m200
    f[dMPM] = R(1) / R(3) * (-R(2) * mxxMyy + mxxMzz + press); // m020
    f[dMMP] = R(1) / R(3) * (mxxMyy - R(2) * mxxMzz + press); // m002
    f[dM00] = m011;
    f[d0M0] = m101;
    f[d00M] = m110;
    const R m4 = press * (R(1) / R(9));
    f[dMPP] = m4;                      // m022
    f[dPMP] = m4;                      // m202
    f[dPPM] = m4;                      // m220
    f[dPPP] = press * (R(1) / R(27));  // m222
    centralMomentsToPopulations(f, vvx, vvy, vvz);
}

// interpolateCF (InterpolationCF.h:57-306) at (x, y, z) in units of the coarse spacing
template <class R>
__host__ __device__ __forceinline__ void interpolateCoarseToFine(R* f, const InterpCoeffs<R>& k, R omegaFine, R x, R y,
                                                                 R z)
{
    const R press = k.d000 + x * k.d100 + y * k.d010 + z * k.d001 + x * y * k.d110 + x * z * k.d101 + y * z * k.d011 +
                    x * y * z * k.d111 + R(3) * x * x * k.LaplaceRho;
    const R vvx = k.a000 + x * k.a100 + y * k.a010 + z * k.a001 + x * x * k.a200 + y * y * k.a020 + z * z * k.a002 +
                  x * y * k.a110 + x * z * k.a101 + y * z * k.a011 + x * y * z * k.a111;
    const R vvy = k.b000 + x * k.b100 + y * k.b010 + z * k.b001 + x * x * k.b200 + y * y * k.b020 + z * z * k.b002 +
                  x * y * k.b110 + x * z * k.b101 + y * z * k.b011 + x * y * z * k.b111;
    const R vvz = k.c000 + x * k.c100 + y * k.c010 + z * k.c001 + x * x * k.c200 + y * y * k.c020 + z * z * k.c002 +
                  x * y * k.c110 + x * z * k.c101 + y * z * k.c011 + x * y * z * k.c111;
    // epsilon (fine / coarse spacing) = 1/2
    const R s = R(1) / R(2) / omegaFine * (R(1) + press);
    const R mxxMyy = -R(2) / R(3) *
                     (k.a100 - k.b010 + R(2) * k.a200 * x - k.b110 * x + k.a110 * y - R(2) * k.b020 * y + k.a101 * z -
                      k.b011 * z - k.b111 * x * z + k.a111 * y * z) *
                     s;
    const R mxxMzz = -R(2) / R(3) *
                     (k.a100 - k.c001 + R(2) * k.a200 * x - k.c101 * x + k.a110 * y - k.c011 * y - k.c111 * x * y +
                      k.a101 * z - R(2) * k.c002 * z + k.a111 * y * z) *
                     s;
    const R m011 = -R(1) / R(3) *
                   (k.b001 + k.c010 + k.b101 * x + k.c110 * x + k.b011 * y + R(2) * k.c020 * y + k.b111 * x * y +
                    R(2) * k.b002 * z + k.c011 * z + k.c111 * x * z) *
                   s;
    const R m101 = -R(1) / R(3) *
                   (k.a001 + k.c100 + k.a101 * x + R(2) * k.c200 * x + k.a011 * y + k.c110 * y + k.a111 * x * y +
                    R(2) * k.a002 * z + k.c101 * z + k.c111 * y * z) *
                   s;
    const R m110 = -R(1) / R(3) *
                   (k.a010 + k.b100 + k.a110 * x + R(2) * k.b200 * x + R(2) * k.a020 * y + k.b110 * y + k.a011 * z +
                    k.b101 * z + k.a111 * x * z + k.b111 * y * z) *
                   s;
    populationsFromMoments(f, press, vvx, vvy, vvz, mxxMyy, mxxMzz, m011, m101, m110);
}

// interpolateFC (InterpolationFC.h:56-263): the coarse node at the cell centre
template <class R>
__host__ __device__ __forceinline__ void interpolateFineToCoarse(R* f, const InterpCoeffs<R>& k, R omegaCoarse)
{
    const R press = k.d000 - R(2) * k.LaplaceRho * (R(1) / R(8));
    // epsilon (coarse / fine spacing) = 2
    const R s = R(2) / omegaCoarse * (R(1) + press);
    const R mxxMyy = -R(2) / R(3) * (k.a100 - k.b010) * s;
    const R mxxMzz = -R(2) / R(3) * (k.a100 - k.c001) * s;
    const R m011 = -R(1) / R(3) * (k.b001 + k.c010) * s;
    const R m101 = -R(1) / R(3) * (k.a001 + k.c100) * s;
    const R m110 = -R(1) / R(3) * (k.a010 + k.b100) * s;
    populationsFromMoments(f, press, k.a000, k.b000, k.c000, mxxMyy, mxxMzz, m011, m101, m110);
}

} // namespace vfb
