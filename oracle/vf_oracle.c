/*
 * vf_oracle.c -- CPU restatement of VirtualFluids' single-GPU LBM time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle that the GPU kernels of
 * virtualfluids_b200 are checked against.  Only tests/, __graft_entry__.smoke()
 * and the cpu_baseline leg of bench.py may load it; the product never does.
 *
 * It restates, in plain C, the arithmetic of the reference's GPU path so that
 * the same sequence of floating point operations is executed for every node:
 *   - D3Q27 direction set and esoteric-twist views
 *       src/lbm/constants/D3Q27.h:46-165,
 *       src/gpu/core/Utilities/KernelUtilities.h:66-125 (twist),
 *       KernelUtilities.h:221-379 (ListIndices, gather/scatter)
 *   - pyramid macroscopic sums   src/lbm/MacroscopicQuantities.h:55-127
 *   - chimera transforms         src/lbm/ChimeraTransformation.h:58-121
 *   - K17 cumulant collision     src/lbm/collision/K17CompressibleNavierStokes.h:87-591
 *   - collision launcher         src/gpu/core/Utilities/RunCollision.cuh:74-143
 *   - BGK compressible           src/gpu/core/Kernel/Compressible/NavierStokes/B92/
 *                                B92CompressibleNavierStokes_Device.cu:41-274
 *   - equilibrium init           src/gpu/core/PreProcessor/PreProcessorStrategy/
 *                                InitNavierStokesCompressible/InitNavierStokesCompressible_Device.cu:44-212
 *   - non-equilibrium init       InitNavierStokesCompressible_Device.cu:216-500
 *   - enstrophy per node         src/gpu/core/PostProcessor/EnstrophyAnalyzer.cu:112-338
 *   - BC formulas                KernelUtilities.h:171-214 and the BC kernels in
 *                                src/gpu/core/BoundaryConditions/{NoSlip,Velocity,Slip,Pressure,Outflow}/
 *
 * Parity is pinned: tests/test_oracle_vs_ref.py compares every function here
 * bit for bit against the reference's own sources compiled on the host
 * (oracle/Makefile, target ref), and tests/golden/ holds fixtures generated
 * from that build so the pin also runs where the reference tree is absent.
 * One function is pinned on the GPU instead: vfo_enstrophy_nodes restates
 * EnstrophyAnalyzer.cu by reading, because that file (a kernel launch and
 * thrust device vectors beside the node function) does not build for the
 * host; tests/test_zy_enstrophy.py compares it with the reference's
 * enstrophyKernel compiled unmodified for sm_100a (oracle/Makefile, target
 * refgpu), and tests/test_enstrophy_host.py against analytic curls.
 *
 * Compiled twice by oracle/Makefile: -DVFO_REAL=double (suffix _f64) and
 * -DVFO_REAL=float (suffix _f32), always with -ffp-contract=off so that no
 * fused multiply-add changes the rounding relative to the reference build.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>

#ifndef VFO_REAL
#define VFO_REAL double
#endif
#ifndef VFO_SUFFIX
#define VFO_SUFFIX _f64
#endif
typedef VFO_REAL real;

/* absolute value in the working precision (std::abs of the reference) */
#define RABS(x) ((real)fabs((double)(x)))

#define VFO_CAT2(a, b) a##b
#define VFO_CAT(a, b) VFO_CAT2(a, b)
#define FN(name) VFO_CAT(name, VFO_SUFFIX)

/* numeric constants are formed in the working precision, as in
 * src/basics/constants/NumericConstants.h:43-290 */
#define C(a, b) ((real)(a) / (real)(b))

/* ------------------------------------------------------------------------ */
/* direction set (src/lbm/constants/D3Q27.h:46-73)                           */
/* ------------------------------------------------------------------------ */
enum {
    d000 = 0, dP00, dM00, d0P0, d0M0, d00P, d00M, dPP0, dMM0, dPM0, dMP0, dP0P, dM0M, dP0M, dM0P,
    d0PP, d0MM, d0PM, d0MP, dPPP, dMPP, dPMP, dMMP, dPPM, dMPM, dPMM, dMMM
};
static const int CX[27] = { 0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1 };
static const int CY[27] = { 0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, -1 };
static const int CZ[27] = { 0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, 1, 1, 1, -1, -1, -1, -1 };
/* inverse direction (D3Q27.h:81-106) */
static const int INV[27] = { 0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17, 26, 25, 24, 23, 22, 21, 20, 19 };

/* lattice weight of a direction: 8/27, 2/27, 1/54, 1/216 by number of
 * non-zero components */
static real weight_of(int d)
{
    int n = (CX[d] != 0) + (CY[d] != 0) + (CZ[d] != 0);
    return n == 0 ? C(8, 27) : n == 1 ? C(2, 27) : n == 2 ? C(1, 54) : C(1, 216);
}

/* c_d . (ux, uy, uz) evaluated left to right over the non-zero components,
 * which is how the reference spells every "vx1 - vx2 + vx3" term. */
static real cdot(int d, real ux, real uy, real uz)
{
    real s = 0;
    int first = 1;
    const int c[3] = { CX[d], CY[d], CZ[d] };
    const real u[3] = { ux, uy, uz };
    for (int a = 0; a < 3; ++a) {
        if (c[a] == 0)
            continue;
        if (first) {
            s = c[a] > 0 ? u[a] : -u[a];
            first = 0;
        } else {
            s = c[a] > 0 ? s + u[a] : s - u[a];
        }
    }
    return s;
}

/* ------------------------------------------------------------------------ */
/* esoteric twist addressing (KernelUtilities.h:66-125, 221-379)             */
/* ------------------------------------------------------------------------ */
/* The eight locations a node touches: bit 0 = shifted along x via neighborX,
 * bit 1 = along y, bit 2 = along z.  neighbor arrays hold the sparse index
 * (+1 shifted) of the next node in the positive axis direction. */
typedef struct { uint32_t k[8]; } locs8;

static locs8 list_indices(uint32_t k, const uint32_t *nx, const uint32_t *ny, const uint32_t *nz)
{
    locs8 L;
    L.k[0] = k;
    L.k[1] = nx[k];
    L.k[2] = ny[k];
    L.k[4] = nz[k];
    L.k[3] = ny[L.k[1]];
    L.k[5] = nz[L.k[1]];
    L.k[6] = nz[L.k[2]];
    L.k[7] = nz[L.k[3]];
    return L;
}

/* location index (0..7) from which direction d is read before collision */
static int loc_of(int d) { return (CX[d] < 0) | ((CY[d] < 0) << 1) | ((CZ[d] < 0) << 2); }

/* array slot of direction d in the even / odd view */
static int slot_of(int d, int isEven) { return isEven ? d : INV[d]; }

static void gather_pre(real f[27], const real *dist, uint64_t N, const locs8 *L, int isEven)
{
    for (int d = 0; d < 27; ++d)
        f[d] = dist[(uint64_t)slot_of(d, isEven) * N + L->k[loc_of(d)]];
}

static void scatter_post(real *dist, uint64_t N, const locs8 *L, int isEven, const real f[27])
{
    for (int d = 0; d < 27; ++d)
        dist[(uint64_t)slot_of(d, isEven) * N + L->k[loc_of(d)]] = f[INV[d]];
}

static void scatter_pre(real *dist, uint64_t N, const locs8 *L, int isEven, const real f[27])
{
    for (int d = 0; d < 27; ++d)
        dist[(uint64_t)slot_of(d, isEven) * N + L->k[loc_of(d)]] = f[d];
}

/* post-collision population moving in direction d at the node */
static real post_value(const real *dist, uint64_t N, const locs8 *L, int isEven, int d)
{
    int e = INV[d];
    return dist[(uint64_t)slot_of(e, isEven) * N + L->k[loc_of(e)]];
}

/* ------------------------------------------------------------------------ */
/* macroscopic sums (MacroscopicQuantities.h:55-127)                          */
/* ------------------------------------------------------------------------ */
static real pyramid_density(const real *f)
{
    real t1 = ((f[dPPP] + f[dMMM]) + (f[dMPM] + f[dPMP])) + ((f[dMPP] + f[dPMM]) + (f[dMMP] + f[dPPM]));
    real t2 = (((f[d0MP] + f[d0PM]) + (f[d0MM] + f[d0PP])) + ((f[dM0P] + f[dP0M]) + (f[dM0M] + f[dP0P]))) +
              ((f[dMP0] + f[dPM0]) + (f[dMM0] + f[dPP0]));
    real t3 = ((f[dM00] + f[dP00]) + (f[d0M0] + f[d0P0])) + (f[d00M] + f[d00P]);
    return ((t1 + t2) + f[d000]) + t3;
}

static real pyramid_jx(const real *f)
{
    return ((((f[dPPP] - f[dMMM]) + (f[dPMP] - f[dMPM])) + ((f[dPMM] - f[dMPP]) + (f[dPPM] - f[dMMP]))) +
            (((f[dP0M] - f[dM0P]) + (f[dP0P] - f[dM0M])) + ((f[dPM0] - f[dMP0]) + (f[dPP0] - f[dMM0])))) +
           (f[dP00] - f[dM00]);
}

static real pyramid_jy(const real *f)
{
    return ((((f[dPPP] - f[dMMM]) + (f[dMPM] - f[dPMP])) + ((f[dMPP] - f[dPMM]) + (f[dPPM] - f[dMMP]))) +
            (((f[d0PM] - f[d0MP]) + (f[d0PP] - f[d0MM])) + ((f[dMP0] - f[dPM0]) + (f[dPP0] - f[dMM0])))) +
           (f[d0P0] - f[d0M0]);
}

static real pyramid_jz(const real *f)
{
    return ((((f[dPPP] - f[dMMM]) + (f[dPMP] - f[dMPM])) + ((f[dMPP] - f[dPMM]) + (f[dMMP] - f[dPPM]))) +
            (((f[d0MP] - f[d0PM]) + (f[d0PP] - f[d0MM])) + ((f[dM0P] - f[dP0M]) + (f[dP0P] - f[dM0M])))) +
           (f[d00P] - f[d00M]);
}

/* ------------------------------------------------------------------------ */
/* chimera transforms (ChimeraTransformation.h:58-121)                        */
/* ------------------------------------------------------------------------ */
static void fwd_k(real *a, real *b, real *c, real vv, real v2, real kinv, real k)
{
    const real m2 = *a + *c;
    const real m1 = *c - *a;
    real m0 = m2 + *b;
    *a = m0;
    m0 *= kinv;
    m0 += (real)1;
    *b = (m1 * kinv - m0 * vv) * k;
    *c = ((m2 - (real)2 * m1 * vv) * kinv + v2 * m0) * k;
}

static void bwd_k(real *a, real *b, real *c, real vv, real v2, real kinv, real k)
{
    const real m0 = (((*c - *b) * C(1, 2) + *b * vv) * kinv + (*a * kinv + (real)1) * (v2 - vv) * C(1, 2)) * k;
    const real m1 = (((*a - *c) - (real)2 * *b * vv) * kinv + (*a * kinv + (real)1) * (-v2)) * k;
    *c = (((*c + *b) * C(1, 2) + *b * vv) * kinv + (*a * kinv + (real)1) * (v2 + vv) * C(1, 2)) * k;
    *a = m0;
    *b = m1;
}

static void fwd_0(real *a, real *b, real *c, real vv, real v2)
{
    const real m1 = (*a + *c) + *b;
    const real m2 = *c - *a;
    *c = (*c + *a) + (v2 * m1 - (real)2 * vv * m2);
    *b = m2 - vv * m1;
    *a = m1;
}

static void bwd_0(real *a, real *b, real *c, real vv, real v2)
{
    const real ma = (*c + *a * (v2 - vv)) * C(1, 2) + *b * (vv - C(1, 2));
    const real mb = ((*a - *c) - *a * v2) - (real)2 * *b * vv;
    *c = (*c + *a * (v2 + vv)) * C(1, 2) + *b * (vv + C(1, 2));
    *b = mb;
    *a = ma;
}

/* One sweep line: the three slots (in the f[] array) that are transformed
 * together and the conditioning pair (Kinverse, K); kn == 0 selects the plain
 * transform.  The tables list the lines of K17CompressibleNavierStokes.h in
 * order: forward z, y, x (:190-222) and backward x, y, z (:525-557). */
typedef struct { int a, b, c, kn, kd; } line_t;

static const line_t FWD_Z[9] = {
    { dMMM, dMM0, dMMP, 36, 1 }, { dM0M, dM00, dM0P, 9, 1 }, { dMPM, dMP0, dMPP, 36, 1 },
    { d0MM, d0M0, d0MP, 9, 1 },  { d00M, d000, d00P, 9, 4 }, { d0PM, d0P0, d0PP, 9, 1 },
    { dPMM, dPM0, dPMP, 36, 1 }, { dP0M, dP00, dP0P, 9, 1 }, { dPPM, dPP0, dPPP, 36, 1 },
};
static const line_t FWD_Y[9] = {
    { dMMM, dM0M, dMPM, 6, 1 }, { dMM0, dM00, dMP0, 0, 0 }, { dMMP, dM0P, dMPP, 18, 1 },
    { d0MM, d00M, d0PM, 3, 2 }, { d0M0, d000, d0P0, 0, 0 }, { d0MP, d00P, d0PP, 9, 2 },
    { dPMM, dP0M, dPPM, 6, 1 }, { dPM0, dP00, dPP0, 0, 0 }, { dPMP, dP0P, dPPP, 18, 1 },
};
/* the last x line uses Kinverse = 3 with K = 1/9, exactly as the reference
 * header does (K17CompressibleNavierStokes.h:222) */
static const line_t FWD_X[9] = {
    { dMMM, d0MM, dPMM, 1, 1 }, { dM0M, d00M, dP0M, 0, 0 }, { dMPM, d0PM, dPPM, 3, 1 },
    { dMM0, d0M0, dPM0, 0, 0 }, { dM00, d000, dP00, 0, 0 }, { dMP0, d0P0, dPP0, 0, 0 },
    { dMMP, d0MP, dPMP, 3, 1 }, { dM0P, d00P, dP0P, 0, 0 }, { dMPP, d0PP, dPPP, -3, 9 },
};

/* moment m_abc lives in the slot of direction (a-1, b-1, c-1) */
#define M(a, b, c) f[mslot[a][b][c]]
static const int mslot[3][3][3] = {
    { { dMMM, dMM0, dMMP }, { dM0M, dM00, dM0P }, { dMPM, dMP0, dMPP } },
    { { d0MM, d0M0, d0MP }, { d00M, d000, d00P }, { d0PM, d0P0, d0PP } },
    { { dPMM, dPM0, dPMP }, { dP0M, dP00, dP0P }, { dPPM, dPP0, dPPP } },
};

static void sweep_fwd(real *f, const line_t *L, real vv, real v2)
{
    for (int i = 0; i < 9; ++i) {
        if (L[i].kn == 0)
            fwd_0(&f[L[i].a], &f[L[i].b], &f[L[i].c], vv, v2);
        else if (L[i].kn < 0) /* Kinverse = -kn, K = 1/kd */
            fwd_k(&f[L[i].a], &f[L[i].b], &f[L[i].c], vv, v2, (real)(-L[i].kn), C(1, L[i].kd));
        else /* Kinverse = kn/kd, K = kd/kn */
            fwd_k(&f[L[i].a], &f[L[i].b], &f[L[i].c], vv, v2, C(L[i].kn, L[i].kd), C(L[i].kd, L[i].kn));
    }
}

/* backward lines in moment coordinates: (a,b,c) index triples along the axis
 * plus the conditioning pair (K17CompressibleNavierStokes.h:525-557) */
typedef struct { int a0, a1, a2, b0, b1, b2, c0, c1, c2, kn, kd; } mline_t;
static const mline_t BWD_X[9] = {
    { 0, 0, 0, 1, 0, 0, 2, 0, 0, 1, 1 }, { 0, 1, 0, 1, 1, 0, 2, 1, 0, 0, 0 }, { 0, 2, 0, 1, 2, 0, 2, 2, 0, 3, 1 },
    { 0, 0, 1, 1, 0, 1, 2, 0, 1, 0, 0 }, { 0, 1, 1, 1, 1, 1, 2, 1, 1, 0, 0 }, { 0, 2, 1, 1, 2, 1, 2, 2, 1, 0, 0 },
    { 0, 0, 2, 1, 0, 2, 2, 0, 2, 3, 1 }, { 0, 1, 2, 1, 1, 2, 2, 1, 2, 0, 0 }, { 0, 2, 2, 1, 2, 2, 2, 2, 2, 9, 1 },
};
static const mline_t BWD_Y[9] = {
    { 0, 0, 0, 0, 1, 0, 0, 2, 0, 6, 1 }, { 0, 0, 1, 0, 1, 1, 0, 2, 1, 0, 0 }, { 0, 0, 2, 0, 1, 2, 0, 2, 2, 18, 1 },
    { 1, 0, 0, 1, 1, 0, 1, 2, 0, 3, 2 }, { 1, 0, 1, 1, 1, 1, 1, 2, 1, 0, 0 }, { 1, 0, 2, 1, 1, 2, 1, 2, 2, 9, 2 },
    { 2, 0, 0, 2, 1, 0, 2, 2, 0, 6, 1 }, { 2, 0, 1, 2, 1, 1, 2, 2, 1, 0, 0 }, { 2, 0, 2, 2, 1, 2, 2, 2, 2, 18, 1 },
};
static const mline_t BWD_Z[9] = {
    { 0, 0, 0, 0, 0, 1, 0, 0, 2, 36, 1 }, { 0, 1, 0, 0, 1, 1, 0, 1, 2, 9, 1 }, { 0, 2, 0, 0, 2, 1, 0, 2, 2, 36, 1 },
    { 1, 0, 0, 1, 0, 1, 1, 0, 2, 9, 1 },  { 1, 1, 0, 1, 1, 1, 1, 1, 2, 9, 4 }, { 1, 2, 0, 1, 2, 1, 1, 2, 2, 9, 1 },
    { 2, 0, 0, 2, 0, 1, 2, 0, 2, 36, 1 }, { 2, 1, 0, 2, 1, 1, 2, 1, 2, 9, 1 }, { 2, 2, 0, 2, 2, 1, 2, 2, 2, 36, 1 },
};

static void sweep_bwd(real *f, const mline_t *L, real vv, real v2)
{
    for (int i = 0; i < 9; ++i) {
        real *a = &M(L[i].a0, L[i].a1, L[i].a2);
        real *b = &M(L[i].b0, L[i].b1, L[i].b2);
        real *c = &M(L[i].c0, L[i].c1, L[i].c2);
        if (L[i].kn == 0)
            bwd_0(a, b, c, vv, v2);
        else
            bwd_k(a, b, c, vv, v2, C(L[i].kn, L[i].kd), C(L[i].kd, L[i].kn));
    }
}

/* the sixth-order central-moment correction, used twice with the same
 * operand order (K17CompressibleNavierStokes.h:320-330 and :489-500) */
static real k17_c222_term(const real *f, real oneOverRho, real drho)
{
    const real m000 = M(0, 0, 0);
    (void)m000;
    const real m111 = M(1, 1, 1), m200 = M(2, 0, 0), m020 = M(0, 2, 0), m002 = M(0, 0, 2);
    const real m022 = M(0, 2, 2), m202 = M(2, 0, 2), m220 = M(2, 2, 0);
    const real m011 = M(0, 1, 1), m101 = M(1, 0, 1), m110 = M(1, 1, 0);
    const real m211 = M(2, 1, 1), m121 = M(1, 2, 1), m112 = M(1, 1, 2);
    const real m120 = M(1, 2, 0), m102 = M(1, 0, 2), m210 = M(2, 1, 0), m012 = M(0, 1, 2);
    const real m201 = M(2, 0, 1), m021 = M(0, 2, 1);
    return (-(real)4 * m111 * m111 - (m200 * m022 + m020 * m202 + m002 * m220) -
            (real)4 * (m011 * m211 + m101 * m121 + m110 * m112) - (real)2 * (m120 * m102 + m210 * m012 + m201 * m021)) *
               oneOverRho +
           ((real)4 * (m101 * m101 * m020 + m011 * m011 * m200 + m110 * m110 * m002) + (real)2 * (m200 * m020 * m002) +
            (real)16 * m110 * m101 * m011) *
               oneOverRho * oneOverRho -
           C(1, 3) * (m022 + m202 + m220) * oneOverRho - C(1, 9) * (m200 + m020 + m002) * oneOverRho +
           ((real)2 * (m101 * m101 + m011 * m011 + m110 * m110) + (m002 * m020 + m002 * m200 + m020 * m200) +
            C(1, 3) * (m002 + m020 + m200)) *
               oneOverRho * oneOverRho * C(2, 3) +
           C(1, 27) * ((drho * drho - drho) * oneOverRho * oneOverRho);
}

/* K17 compressible cumulant collision on one node, in place on f[27]
 * (K17CompressibleNavierStokes.h:87-591, TurbulenceModel::None). */
void FN(vfo_k17_collide)(real *f, real omega, const real *limiter, real fx, real fy, real fz, real *out_rho,
                         real *out_vx, real *out_vy, real *out_vz)
{
    const real drho = pyramid_density(f);
    const real oneOverRho = (real)1 / (drho + (real)1);
    real vvx = pyramid_jx(f) * oneOverRho;
    real vvy = pyramid_jy(f) * oneOverRho;
    real vvz = pyramid_jz(f) * oneOverRho;
    vvx += fx;
    vvy += fy;
    vvz += fz;
    const real vx2 = vvx * vvx, vy2 = vvy * vvy, vz2 = vvz * vvz;
    const real qlP = limiter[0], qlM = limiter[1], qlD = limiter[2];

    sweep_fwd(f, FWD_Z, vvz, vz2);
    sweep_fwd(f, FWD_Y, vvy, vy2);
    sweep_fwd(f, FWD_X, vvx, vx2);

    /* relaxation rates (:245-273) */
    const real OxxPyyPzz = (real)1;
    const real OxyyPxzz = (real)8 * (-(real)2 + omega) * ((real)1 + (real)2 * omega) /
                          (-(real)8 - (real)14 * omega + (real)7 * omega * omega);
    const real OxyyMxzz = (real)8 * (-(real)2 + omega) * (-(real)7 + (real)4 * omega) /
                          ((real)56 - (real)50 * omega + (real)9 * omega * omega);
    const real Oxyz = (real)24 * (-(real)2 + omega) * (-(real)2 - (real)7 * omega + (real)3 * omega * omega) /
                      ((real)48 + (real)152 * omega - (real)130 * omega * omega + (real)29 * omega * omega * omega);
    const real O4 = (real)1, O5 = (real)1, O6 = (real)1;
    const real factorA = ((real)4 + (real)2 * omega - (real)3 * omega * omega) /
                         ((real)2 - (real)7 * omega + (real)5 * omega * omega);
    const real factorB = ((real)4 + (real)28 * omega - (real)14 * omega * omega) /
                         ((real)6 - (real)21 * omega + (real)15 * omega * omega);

    /* cumulants of order 4..6 (:282-316) */
    real cm211 = M(2, 1, 1) - ((M(2, 0, 0) + C(1, 3)) * M(0, 1, 1) + (real)2 * M(1, 1, 0) * M(1, 0, 1)) * oneOverRho;
    real cm121 = M(1, 2, 1) - ((M(0, 2, 0) + C(1, 3)) * M(1, 0, 1) + (real)2 * M(1, 1, 0) * M(0, 1, 1)) * oneOverRho;
    real cm112 = M(1, 1, 2) - ((M(0, 0, 2) + C(1, 3)) * M(1, 1, 0) + (real)2 * M(1, 0, 1) * M(0, 1, 1)) * oneOverRho;
    real cm220 = M(2, 2, 0) - (((M(2, 0, 0) * M(0, 2, 0) + (real)2 * M(1, 1, 0) * M(1, 1, 0)) + C(1, 3) * (M(2, 0, 0) + M(0, 2, 0))) * oneOverRho -
                               C(1, 9) * (drho * oneOverRho));
    real cm202 = M(2, 0, 2) - (((M(2, 0, 0) * M(0, 0, 2) + (real)2 * M(1, 0, 1) * M(1, 0, 1)) + C(1, 3) * (M(2, 0, 0) + M(0, 0, 2))) * oneOverRho -
                               C(1, 9) * (drho * oneOverRho));
    real cm022 = M(0, 2, 2) - (((M(0, 0, 2) * M(0, 2, 0) + (real)2 * M(0, 1, 1) * M(0, 1, 1)) + C(1, 3) * (M(0, 0, 2) + M(0, 2, 0))) * oneOverRho -
                               C(1, 9) * (drho * oneOverRho));
    real cm122 = M(1, 2, 2) - ((M(0, 0, 2) * M(1, 2, 0) + M(0, 2, 0) * M(1, 0, 2) + (real)4 * M(0, 1, 1) * M(1, 1, 1) +
                                (real)2 * (M(1, 0, 1) * M(0, 2, 1) + M(1, 1, 0) * M(0, 1, 2))) +
                               C(1, 3) * (M(1, 2, 0) + M(1, 0, 2))) * oneOverRho;
    real cm212 = M(2, 1, 2) - ((M(0, 0, 2) * M(2, 1, 0) + M(2, 0, 0) * M(0, 1, 2) + (real)4 * M(1, 0, 1) * M(1, 1, 1) +
                                (real)2 * (M(0, 1, 1) * M(2, 0, 1) + M(1, 1, 0) * M(1, 0, 2))) +
                               C(1, 3) * (M(2, 1, 0) + M(0, 1, 2))) * oneOverRho;
    real cm221 = M(2, 2, 1) - ((M(2, 0, 0) * M(0, 2, 1) + M(0, 2, 0) * M(2, 0, 1) + (real)4 * M(1, 1, 0) * M(1, 1, 1) +
                                (real)2 * (M(1, 0, 1) * M(1, 2, 0) + M(0, 1, 1) * M(2, 1, 0))) +
                               C(1, 3) * (M(0, 2, 1) + M(2, 0, 1))) * oneOverRho;
    real cm222 = M(2, 2, 2) + k17_c222_term(f, oneOverRho, drho);

    /* second and third order combinations (:329-346) */
    real mxxPyyPzz = M(2, 0, 0) + M(0, 2, 0) + M(0, 0, 2);
    real mxxMyy = M(2, 0, 0) - M(0, 2, 0);
    real mxxMzz = M(2, 0, 0) - M(0, 0, 2);
    real mxxyPyzz = M(2, 1, 0) + M(0, 1, 2);
    real mxxyMyzz = M(2, 1, 0) - M(0, 1, 2);
    real mxxzPyyz = M(2, 0, 1) + M(0, 2, 1);
    real mxxzMyyz = M(2, 0, 1) - M(0, 2, 1);
    real mxyyPxzz = M(1, 2, 0) + M(1, 0, 2);
    real mxyyMxzz = M(1, 2, 0) - M(1, 0, 2);

    /* velocity gradients (:357-362) */
    const real Dxy = -(real)3 * omega * M(1, 1, 0);
    const real Dxz = -(real)3 * omega * M(1, 0, 1);
    const real Dyz = -(real)3 * omega * M(0, 1, 1);
    const real dxux = C(1, 2) * (-omega) * (mxxMyy + mxxMzz) + C(1, 2) * OxxPyyPzz * (M(0, 0, 0) - mxxPyyPzz);
    const real dyuy = dxux + omega * C(3, 2) * mxxMyy;
    const real dzuz = dxux + omega * C(3, 2) * mxxMzz;

    /* second order relaxation with correction (:387-389) */
    mxxPyyPzz += OxxPyyPzz * (M(0, 0, 0) - mxxPyyPzz) -
                 (real)3 * ((real)1 - C(1, 2) * OxxPyyPzz) * (vx2 * dxux + vy2 * dyuy + vz2 * dzuz);
    mxxMyy += omega * (-mxxMyy) - (real)3 * ((real)1 + C(1, 2) * (-omega)) * (vx2 * dxux - vy2 * dyuy);
    mxxMzz += omega * (-mxxMzz) - (real)3 * ((real)1 + C(1, 2) * (-omega)) * (vx2 * dxux - vz2 * dzuz);
    M(0, 1, 1) += omega * (-M(0, 1, 1));
    M(1, 0, 1) += omega * (-M(1, 0, 1));
    M(1, 1, 0) += omega * (-M(1, 1, 0));

    /* third order with quartic limiter (:404-417) */
    real w;
    w = Oxyz + ((real)1 - Oxyz) * RABS(M(1, 1, 1)) / (RABS(M(1, 1, 1)) + qlD);
    M(1, 1, 1) += w * (-M(1, 1, 1));
    w = OxyyPxzz + ((real)1 - OxyyPxzz) * RABS(mxxyPyzz) / (RABS(mxxyPyzz) + qlP);
    mxxyPyzz += w * (-mxxyPyzz);
    w = OxyyMxzz + ((real)1 - OxyyMxzz) * RABS(mxxyMyzz) / (RABS(mxxyMyzz) + qlM);
    mxxyMyzz += w * (-mxxyMyzz);
    w = OxyyPxzz + ((real)1 - OxyyPxzz) * RABS(mxxzPyyz) / (RABS(mxxzPyyz) + qlP);
    mxxzPyyz += w * (-mxxzPyyz);
    w = OxyyMxzz + ((real)1 - OxyyMxzz) * RABS(mxxzMyyz) / (RABS(mxxzMyyz) + qlM);
    mxxzMyyz += w * (-mxxzMyyz);
    w = OxyyPxzz + ((real)1 - OxyyPxzz) * RABS(mxyyPxzz) / (RABS(mxyyPxzz) + qlP);
    mxyyPxzz += w * (-mxyyPxzz);
    w = OxyyMxzz + ((real)1 - OxyyMxzz) * RABS(mxyyMxzz) / (RABS(mxyyMxzz) + qlM);
    mxyyMxzz += w * (-mxyyMxzz);

    /* back to single moments (:431-441) */
    M(2, 0, 0) = C(1, 3) * (mxxMyy + mxxMzz + mxxPyyPzz);
    M(0, 2, 0) = C(1, 3) * (-(real)2 * mxxMyy + mxxMzz + mxxPyyPzz);
    M(0, 0, 2) = C(1, 3) * (mxxMyy - (real)2 * mxxMzz + mxxPyyPzz);
    M(2, 1, 0) = (mxxyMyzz + mxxyPyzz) * C(1, 2);
    M(0, 1, 2) = (-mxxyMyzz + mxxyPyzz) * C(1, 2);
    M(2, 0, 1) = (mxxzMyyz + mxxzPyyz) * C(1, 2);
    M(0, 2, 1) = (-mxxzMyyz + mxxzPyyz) * C(1, 2);
    M(1, 2, 0) = (mxyyMxzz + mxyyPxzz) * C(1, 2);
    M(1, 0, 2) = (-mxyyMxzz + mxyyPxzz) * C(1, 2);

    /* fourth order to modified equilibrium; fifth and sixth to zero (:452-471) */
    cm022 = -O4 * ((real)1 / omega - C(1, 2)) * (dyuy + dzuz) * C(2, 3) * factorA + ((real)1 - O4) * (cm022);
    cm202 = -O4 * ((real)1 / omega - C(1, 2)) * (dxux + dzuz) * C(2, 3) * factorA + ((real)1 - O4) * (cm202);
    cm220 = -O4 * ((real)1 / omega - C(1, 2)) * (dyuy + dxux) * C(2, 3) * factorA + ((real)1 - O4) * (cm220);
    cm112 = -O4 * ((real)1 / omega - C(1, 2)) * Dxy * C(1, 3) * factorB + ((real)1 - O4) * (cm112);
    cm121 = -O4 * ((real)1 / omega - C(1, 2)) * Dxz * C(1, 3) * factorB + ((real)1 - O4) * (cm121);
    cm211 = -O4 * ((real)1 / omega - C(1, 2)) * Dyz * C(1, 3) * factorB + ((real)1 - O4) * (cm211);
    cm122 += O5 * (-cm122);
    cm212 += O5 * (-cm212);
    cm221 += O5 * (-cm221);
    cm222 += O6 * (-cm222);

    /* cumulants back to central moments (:478-505) */
    M(2, 1, 1) = cm211 + C(1, 3) * (((real)3 * M(2, 0, 0) + (real)1) * M(0, 1, 1) + (real)6 * M(1, 1, 0) * M(1, 0, 1)) * oneOverRho;
    M(1, 2, 1) = cm121 + C(1, 3) * (((real)3 * M(0, 2, 0) + (real)1) * M(1, 0, 1) + (real)6 * M(1, 1, 0) * M(0, 1, 1)) * oneOverRho;
    M(1, 1, 2) = cm112 + C(1, 3) * (((real)3 * M(0, 0, 2) + (real)1) * M(1, 1, 0) + (real)6 * M(1, 0, 1) * M(0, 1, 1)) * oneOverRho;
    M(2, 2, 0) = cm220 + (((M(2, 0, 0) * M(0, 2, 0) + (real)2 * M(1, 1, 0) * M(1, 1, 0)) * (real)9 + (real)3 * (M(2, 0, 0) + M(0, 2, 0))) * oneOverRho -
                          (drho * oneOverRho)) * C(1, 9);
    M(2, 0, 2) = cm202 + (((M(2, 0, 0) * M(0, 0, 2) + (real)2 * M(1, 0, 1) * M(1, 0, 1)) * (real)9 + (real)3 * (M(2, 0, 0) + M(0, 0, 2))) * oneOverRho -
                          (drho * oneOverRho)) * C(1, 9);
    M(0, 2, 2) = cm022 + (((M(0, 0, 2) * M(0, 2, 0) + (real)2 * M(0, 1, 1) * M(0, 1, 1)) * (real)9 + (real)3 * (M(0, 0, 2) + M(0, 2, 0))) * oneOverRho -
                          (drho * oneOverRho)) * C(1, 9);
    M(1, 2, 2) = cm122 + C(1, 3) *
                             ((real)3 * (M(0, 0, 2) * M(1, 2, 0) + M(0, 2, 0) * M(1, 0, 2) + (real)4 * M(0, 1, 1) * M(1, 1, 1) +
                                         (real)2 * (M(1, 0, 1) * M(0, 2, 1) + M(1, 1, 0) * M(0, 1, 2))) +
                              (M(1, 2, 0) + M(1, 0, 2))) * oneOverRho;
    M(2, 1, 2) = cm212 + C(1, 3) *
                             ((real)3 * (M(0, 0, 2) * M(2, 1, 0) + M(2, 0, 0) * M(0, 1, 2) + (real)4 * M(1, 0, 1) * M(1, 1, 1) +
                                         (real)2 * (M(0, 1, 1) * M(2, 0, 1) + M(1, 1, 0) * M(1, 0, 2))) +
                              (M(2, 1, 0) + M(0, 1, 2))) * oneOverRho;
    M(2, 2, 1) = cm221 + C(1, 3) *
                             ((real)3 * (M(2, 0, 0) * M(0, 2, 1) + M(0, 2, 0) * M(2, 0, 1) + (real)4 * M(1, 1, 0) * M(1, 1, 1) +
                                         (real)2 * (M(1, 0, 1) * M(1, 2, 0) + M(0, 1, 1) * M(2, 1, 0))) +
                              (M(0, 2, 1) + M(2, 0, 1))) * oneOverRho;
    M(2, 2, 2) = cm222 - k17_c222_term(f, oneOverRho, drho);

    /* first moments flip sign (force, :512-514) */
    M(1, 0, 0) = -M(1, 0, 0);
    M(0, 1, 0) = -M(0, 1, 0);
    M(0, 0, 1) = -M(0, 0, 1);

    sweep_bwd(f, BWD_X, vvx, vx2);
    sweep_bwd(f, BWD_Y, vvy, vy2);
    sweep_bwd(f, BWD_Z, vvz, vz2);

    if (out_rho) *out_rho = drho;
    if (out_vx) *out_vx = vvx;
    if (out_vy) *out_vy = vvy;
    if (out_vz) *out_vz = vvz;
}
#undef M

/* ------------------------------------------------------------------------ */
/* collision over a fluid-node list (RunCollision.cuh:74-143)                 */
/* ------------------------------------------------------------------------ */
/* flags: bit 0 = write macroscopic values, bit 1 = apply per-node body force */
void FN(vfo_collision_k17)(real *dist, uint64_t N, const uint32_t *nx, const uint32_t *ny, const uint32_t *nz,
                           const uint32_t *fluidNodes, uint32_t nFluid, real omega, const real *forces,
                           real forceFactor, const real *limiters, int isEven, int flags, real *rho, real *vx,
                           real *vy, real *vz, real *bodyFx, real *bodyFy, real *bodyFz)
{
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)nFluid; ++i) {
        const uint32_t k = fluidNodes[i];
        real fx, fy, fz;
        if (flags & 2) {
            fx = (forces[0] + bodyFx[k]) * C(1, 2) * forceFactor;
            fy = (forces[1] + bodyFy[k]) * C(1, 2) * forceFactor;
            fz = (forces[2] + bodyFz[k]) * C(1, 2) * forceFactor;
            bodyFx[k] = 0;
            bodyFy[k] = 0;
            bodyFz[k] = 0;
        } else {
            fx = forces[0] * C(1, 2) * forceFactor;
            fy = forces[1] * C(1, 2) * forceFactor;
            fz = forces[2] * C(1, 2) * forceFactor;
        }
        locs8 L = list_indices(k, nx, ny, nz);
        real f[27];
        gather_pre(f, dist, N, &L, isEven);
        real r, ux, uy, uz;
        FN(vfo_k17_collide)(f, omega, limiters, fx, fy, fz, &r, &ux, &uy, &uz);
        if (flags & 1) {
            vx[k] = ux;
            vy[k] = uy;
            vz[k] = uz;
            rho[k] = r;
        }
        scatter_post(dist, N, &L, isEven, f);
    }
}

/* ------------------------------------------------------------------------ */
/* BGK compressible (B92CompressibleNavierStokes_Device.cu:41-274)            */
/* ------------------------------------------------------------------------ */
#define GEO_SOLID 15
#define GEO_VOID 16

void FN(vfo_bgk_collide)(real *f, real omega)
{
    /* pair sums in the order of B92CompressibleNavierStokes_Device.cu:194 */
    static const int pairs[13][2] = {
        { dPPP, dMMM }, { dMMP, dPPM }, { dPMP, dMPM }, { dMPP, dPMM }, { dPP0, dMM0 }, { dMP0, dPM0 }, { dP0P, dM0M },
        { dP0M, dM0P }, { d0PP, d0MM }, { d0PM, d0MP }, { dP00, dM00 }, { d0P0, d0M0 }, { d00P, d00M },
    };
    real drho = f[pairs[0][0]] + f[pairs[0][1]];
    for (int i = 1; i < 13; ++i)
        drho = drho + (f[pairs[i][0]] + f[pairs[i][1]]);
    drho = drho + f[d000];
    const real rho = drho + (real)1;
    const real OORho = (real)1 / rho;
    /* momentum differences (:197-199) */
    static const int jx[9][2] = { { dPPP, dMMM }, { dPPM, dMMP }, { dPMP, dMPM }, { dPMM, dMPP }, { dPP0, dMM0 },
                                  { dPM0, dMP0 }, { dP0P, dM0M }, { dP0M, dM0P }, { dP00, dM00 } };
    static const int jy[9][2] = { { dPPP, dMMM }, { dPPM, dMMP }, { dMPM, dPMP }, { dMPP, dPMM }, { dPP0, dMM0 },
                                  { dMP0, dPM0 }, { d0PP, d0MM }, { d0PM, d0MP }, { d0P0, d0M0 } };
    static const int jz[9][2] = { { dPPP, dMMM }, { dMMP, dPPM }, { dPMP, dMPM }, { dMPP, dPMM }, { dP0P, dM0M },
                                  { dM0P, dP0M }, { d0PP, d0MM }, { d0MP, d0PM }, { d00P, d00M } };
    real sx = f[jx[0][0]] - f[jx[0][1]], sy = f[jy[0][0]] - f[jy[0][1]], sz = f[jz[0][0]] - f[jz[0][1]];
    for (int i = 1; i < 9; ++i) {
        sx = sx + (f[jx[i][0]] - f[jx[i][1]]);
        sy = sy + (f[jy[i][0]] - f[jy[i][1]]);
        sz = sz + (f[jz[i][0]] - f[jz[i][1]]);
    }
    const real vx1 = OORho * sx, vx2 = OORho * sy, vx3 = OORho * sz;
    const real cusq = C(3, 2) * (vx1 * vx1 + vx2 * vx2 + vx3 * vx3);
    /* relaxation (:206-234) */
    f[d000] = f[d000] * ((real)1 + (-omega)) - (-omega) * C(8, 27) * (drho - rho * cusq);
    for (int d = 1; d < 27; ++d) {
        const real cu = cdot(d, vx1, vx2, vx3);
        f[d] = f[d] * ((real)1 + (-omega)) -
               (-omega) * weight_of(d) * (drho + rho * ((real)3 * (cu) + C(9, 2) * (cu) * (cu) - cusq));
    }
}

/* BGK over all nodes with a geometry check; isEven selects the view */
void FN(vfo_collision_bgk)(real *dist, uint64_t N, const uint32_t *geo, const uint32_t *nx, const uint32_t *ny,
                           const uint32_t *nz, real omega, int isEven)
{
#pragma omp parallel for schedule(static)
    for (long long kk = 0; kk < (long long)N; ++kk) {
        const uint32_t k = (uint32_t)kk;
        if (geo[k] == GEO_SOLID || geo[k] == GEO_VOID)
            continue;
        locs8 L = list_indices(k, nx, ny, nz);
        real f[27];
        gather_pre(f, dist, N, &L, isEven);
        FN(vfo_bgk_collide)(f, omega);
        scatter_post(dist, N, &L, isEven, f);
    }
}

/* ------------------------------------------------------------------------ */
/* equilibrium init (InitNavierStokesCompressible_Device.cu:44-212)           */
/* ------------------------------------------------------------------------ */
static real feq_full(int d, real drho, real vx1, real vx2, real vx3, real cu_sq)
{
    if (d == d000)
        return C(8, 27) * (drho - cu_sq * ((real)1 + drho));
    const real cu = cdot(d, vx1, vx2, vx3);
    return weight_of(d) * (drho + ((real)1 + drho) * ((real)3 * (cu) + C(9, 2) * (cu) * (cu) - cu_sq));
}

void FN(vfo_init_eq)(real *dist, uint64_t N, const uint32_t *geo, const uint32_t *nx, const uint32_t *ny,
                     const uint32_t *nz, const real *rho, const real *ux, const real *uy, const real *uz, int isEven)
{
    for (uint64_t kk = 0; kk < N; ++kk) {
        const uint32_t k = (uint32_t)kk;
        if (geo[k] == GEO_SOLID || geo[k] == GEO_VOID)
            continue;
        const real drho = rho[k], vx1 = ux[k], vx2 = uy[k], vx3 = uz[k];
        const real cu_sq = C(3, 2) * (vx1 * vx1 + vx2 * vx2 + vx3 * vx3);
        locs8 L = list_indices(k, nx, ny, nz);
        real f[27];
        for (int d = 0; d < 27; ++d)
            f[d] = feq_full(d, drho, vx1, vx2, vx3, cu_sq);
        scatter_pre(dist, N, &L, isEven, f);
    }
}

/* ------------------------------------------------------------------------ */
/* non-equilibrium init (InitNavierStokesCompressible_Device.cu:216-500)     */
/* ------------------------------------------------------------------------ */
/* Coefficient slot of each direction: opposite directions share one
 * non-equilibrium value (:460-486).  Slots: 0 rest, 1-3 the x, y, z axes,
 * 4 xy same sign, 5 xy opposite, 6 xz same, 7 xz opposite, 8 yz same,
 * 9 yz opposite, 10 PPP/MMM, 11 PPM/MMP, 12 PMP/MPM, 13 PMM/MPP. */
static const int NEQ_SLOT[27] = { 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 8, 8, 9, 9, 10, 13, 12, 11, 11, 12, 13, 10 };

/* The fourteen non-equilibrium coefficients from the central-difference
 * velocity gradient g[a][b] = d u_a / d x_b (:378-425, the strain part of the
 * Chapman-Enskog expansion at first order).  The reference spells them with
 * double literals, so every product with a literal is formed in double even
 * when real is float, while sums of two gradients in parentheses stay in real;
 * each coefficient is rounded to real once.  Its factors eps_new and op are 1
 * and multiply exactly; they are left out. */
static void noneq_coefficients(const real g[3][3], real omega, real c[14])
{
    const real ax = g[0][0], ay = g[0][1], az = g[0][2];
    const real bx = g[1][0], by = g[1][1], bz = g[1][2];
    const real cx = g[2][0], cy = g[2][1], cz = g[2][2];
    const real o = omega;
    c[1] = (real)((5. * ax * o + 5. * by * o + 5. * cz * o - 8. * ax + 4. * by + 4. * cz) / (54. * o));
    c[2] = (real)(c[1] + (2. * (ax - by)) / (9. * o));
    c[3] = (real)(c[1] + (2. * (ax - cz)) / (9. * o));
    c[4] = (real)(-(5. * cz * o + 3. * (ay + bx) - 2. * cz + ax * (5. * o + 1.) + by * (5. * o + 1.)) / (54. * o));
    c[5] = (real)(c[4] + (ay + bx) / (9. * o));
    c[6] = (real)(-(5. * cz * o + by * (5. * o - 2.) + 3. * (az + cx) + cz + ax * (5. * o + 1.)) / (54. * o));
    c[7] = (real)(c[6] + (az + cx) / (9. * o));
    c[8] = (real)(-(5. * ax * o + 5. * by * o + 5. * cz * o - 2. * ax + by + 3. * bz + 3. * cy + cz) / (54. * o));
    c[9] = (real)(c[8] + (bz + cy) / (9. * o));
    c[0] = (real)((5. * (ax + by + cz)) / 9.);
    c[10] = (real)(-(ay + az + bx + bz + cx + cy) / (72. * o));
    c[11] = (real)(-c[10] - (ay + bx) / (36. * o));
    c[12] = (real)(-c[10] - (az + cx) / (36. * o));
    c[13] = (real)(-c[10] - (bz + cy) / (36. * o));
}

/* one node: equilibrium of (drho, u) plus (1 + drho) times the coefficient of
 * each direction's slot (:428-486), in canonical direction order */
void FN(vfo_noneq_node)(real drho, real vx1, real vx2, real vx3, const real *grad9, real omega, real *f)
{
    real g[3][3], c[14];
    for (int a = 0; a < 9; ++a)
        g[a / 3][a % 3] = grad9[a];
    noneq_coefficients(g, omega, c);
    const real cu_sq = C(3, 2) * (vx1 * vx1 + vx2 * vx2 + vx3 * vx3);
    for (int d = 0; d < 27; ++d) {
        const real eq = feq_full(d, drho, vx1, vx2, vx3, cu_sq);
        f[d] = eq + ((real)1 + drho) * c[NEQ_SLOT[d]];
    }
}

void FN(vfo_init_noneq)(real *dist, uint64_t N, const uint32_t *geo, const uint32_t *nx, const uint32_t *ny,
                        const uint32_t *nz, const uint32_t *nneg, const real *rho, const real *ux, const real *uy,
                        const real *uz, real omega, int isEven)
{
    const real *u[3] = { ux, uy, uz };
    for (uint64_t kk = 0; kk < N; ++kk) {
        const uint32_t k = (uint32_t)kk;
        if (geo[k] == GEO_SOLID || geo[k] == GEO_VOID) {
            dist[k] = (real)96; /* the rest population of a solid node is set to 96 (:490-499) */
            continue;
        }
        /* axis neighbours; the negative ones through the inverse (-x-y-z)
         * neighbour and two positive steps (:347-353) */
        const uint32_t w = nneg[k];
        const uint32_t plus[3] = { nx[k], ny[k], nz[k] };
        const uint32_t minus[3] = { nz[ny[w]], nz[nx[w]], ny[nx[w]] };
        real grad[9];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                grad[3 * a + b] = (u[a][plus[b]] - u[a][minus[b]]) / (real)2;
        real f[27];
        FN(vfo_noneq_node)(rho[k], ux[k], uy[k], uz[k], grad, omega, f);
        locs8 L = list_indices(k, nx, ny, nz);
        scatter_pre(dist, N, &L, isEven, f);
    }
}

/* ------------------------------------------------------------------------ */
/* boundary conditions                                                        */
/* ------------------------------------------------------------------------ */
/* macroscopic values from post-collision populations with the plain sums of
 * NoSlipInterpolatedCompressible.cu:144-160 (shared by the velocity and slip
 * kernels).  g[d] is the post-collision population moving in direction d. */
static void bc_macros(const real *g, real *drho, real *vx1, real *vx2, real *vx3)
{
    static const int order[27] = { dPMP, dMPP, dPPP, dMMP, dPMM, dMPM, dPPM, dMMM, d0PM, d0MP, d0PP, d0MM, dP0M, dM0P,
                                   dP0P, dM0M, dPM0, dMP0, dPP0, dMM0, d00P, d00M, d0P0, d0M0, dP00, dM00, d000 };
    real s = g[order[0]];
    for (int i = 1; i < 27; ++i)
        s = s + g[order[i]];
    *drho = s;
    const real r1 = (real)1 + s;
    *vx1 = (((g[dPMP] - g[dMPM]) - (g[dMPP] - g[dPMM])) + ((g[dPPP] - g[dMMM]) - (g[dMMP] - g[dPPM])) +
            ((g[dP0M] - g[dM0P]) + (g[dP0P] - g[dM0M])) + ((g[dPM0] - g[dMP0]) + (g[dPP0] - g[dMM0])) +
            (g[dP00] - g[dM00])) / r1;
    *vx2 = ((-(g[dPMP] - g[dMPM]) + (g[dMPP] - g[dPMM])) + ((g[dPPP] - g[dMMM]) - (g[dMMP] - g[dPPM])) +
            ((g[d0PM] - g[d0MP]) + (g[d0PP] - g[d0MM])) + (-(g[dPM0] - g[dMP0]) + (g[dPP0] - g[dMM0])) +
            (g[d0P0] - g[d0M0])) / r1;
    *vx3 = (((g[dPMP] - g[dMPM]) + (g[dMPP] - g[dPMM])) + ((g[dPPP] - g[dMMM]) + (g[dMMP] - g[dPPM])) +
            (-(g[d0PM] - g[d0MP]) + (g[d0PP] - g[d0MM])) + ((g[dP0P] - g[dM0M]) - (g[dP0M] - g[dM0P])) +
            (g[d00P] - g[d00M])) / r1;
}

/* KernelUtilities.h:171-174 */
static real feq_bc(real drho, real vel, real cu_sq, real w)
{
    return w * (drho + C(9, 2) * vel * vel * ((real)1 + drho) - cu_sq);
}
/* KernelUtilities.h:189-195 */
static real interp_noslip(real q, real f, real finv, real feq, real omega)
{
    return ((real)1 - q) / ((real)1 + q) * (f - finv + (f + finv - (real)2 * feq * omega) / ((real)1 - omega)) * C(1, 2) +
           (q * (f + finv)) / ((real)1 + q);
}
/* KernelUtilities.h:176-182 */
static real interp_velo(real q, real f, real finv, real feq, real omega, real vel, real w)
{
    return ((real)1 - q) / ((real)1 + q) * (f - finv + (f + finv - (real)2 * feq * omega) / ((real)1 - omega)) * C(1, 2) +
           (q * (f + finv) - (real)6 * w * vel) / ((real)1 + q);
}

/* q directions in the order the BC kernels visit them */
static const int QORDER[26] = { dP00, dM00, d0P0, d0M0, d00P, d00M, dPP0, dMM0, dPM0, dMP0, dP0P, dM0M, dP0M,
                                dM0P, d0PP, d0MM, d0PM, d0MP, dPPP, dMMM, dPPM, dMMP, dPMP, dMPM, dPMM, dMPP };

#define BC_NOSLIP_INTERP 0
#define BC_NOSLIP_BB 1
#define BC_VELOCITY_INTERP 2
#define BC_VELOCITY_BB 3
#define BC_SLIP 4
#define BC_VELOCITY_PRESSURE 5

/* post-collision BC over a compacted list (kind selects the formula):
 *   NoSlipInterpolatedCompressible.cu:44-378, NoSlipBounceBack.cu,
 *   VelocityInterpolatedCompressible.cu:44-418, VelocityBounceBack.cu,
 *   SlipCompressible.cu:45-550.
 * q is direction-major: q[d * nBC + i]; velocities are per BC node. */
void FN(vfo_bc_post)(int kind, real *dist, uint64_t N, const uint32_t *nx, const uint32_t *ny, const uint32_t *nz,
                     const int32_t *bcNodes, const real *q, uint32_t nBC, real omega, const real *Vx, const real *Vy,
                     const real *Vz, int isEven)
{
    for (uint32_t i = 0; i < nBC; ++i) {
        const locs8 L = list_indices((uint32_t)bcNodes[i], nx, ny, nz);
        real g[27];
        for (int d = 0; d < 27; ++d)
            g[d] = post_value(dist, N, &L, isEven, d);
        real drho = 0, vx1 = 0, vx2 = 0, vx3 = 0, cu_sq = 0;
        if (kind == BC_NOSLIP_INTERP || kind == BC_VELOCITY_INTERP || kind == BC_SLIP || kind == BC_VELOCITY_PRESSURE) {
            bc_macros(g, &drho, &vx1, &vx2, &vx3);
            cu_sq = C(3, 2) * (vx1 * vx1 + vx2 * vx2 + vx3 * vx3) * ((real)1 + drho);
        }
        real UX = 0, UY = 0, UZ = 0;
        if (kind == BC_VELOCITY_INTERP || kind == BC_VELOCITY_BB || kind == BC_VELOCITY_PRESSURE) {
            UX = Vx[i];
            UY = Vy[i];
            UZ = Vz[i];
        }
        int flag[3] = { 0, 0, 0 };
        const int odd = !isEven;
        for (int j = 0; j < 26; ++j) {
            const int d = QORDER[j];
            const real qd = q[(uint64_t)d * nBC + i];
            if (!(qd >= (real)0 && qd <= (real)1))
                continue;
            const int e = INV[d];
            real *target = &dist[(uint64_t)slot_of(e, odd) * N + L.k[loc_of(e)]];
            const real w = weight_of(d);
            switch (kind) {
            case BC_NOSLIP_BB:
                *target = g[d];
                break;
            case BC_VELOCITY_BB: {
                /* 6 w (-c_d . U) with 6w = 4/9, 1/9, 1/36 */
                const int n = (CX[d] != 0) + (CY[d] != 0) + (CZ[d] != 0);
                const real k6 = n == 1 ? C(4, 9) : n == 2 ? C(1, 9) : C(1, 36);
                *target = g[d] + k6 * cdot(e, UX, UY, UZ);
                break;
            }
            case BC_NOSLIP_INTERP: {
                const real feq = feq_bc(drho, cdot(d, vx1, vx2, vx3), cu_sq, w);
                *target = interp_noslip(qd, g[d], g[e], feq, omega);
                break;
            }
            case BC_VELOCITY_INTERP: {
                const real feq = feq_bc(drho, cdot(d, vx1, vx2, vx3), cu_sq, w);
                *target = interp_velo(qd, g[d], g[e], feq, omega, cdot(d, UX, UY, UZ), w);
                break;
            }
            case BC_VELOCITY_PRESSURE: {
                /* the velocity formula minus w drho (KernelUtilities.h:208-214,
                 * VelocityWithPressureInterpolatedCompressible.cu) */
                const real feq = feq_bc(drho, cdot(d, vx1, vx2, vx3), cu_sq, w);
                *target = interp_velo(qd, g[d], g[e], feq, omega, cdot(d, UX, UY, UZ), w) - w * drho;
                break;
            }
            case BC_SLIP: {
                /* the normal velocity components are zeroed for every axis
                 * that has an active axis direction (SlipCompressible.cu) */
                const int n = (CX[d] != 0) + (CY[d] != 0) + (CZ[d] != 0);
                if (n == 1) {
                    flag[CX[d] != 0 ? 0 : CY[d] != 0 ? 1 : 2] = 1;
                }
                const real sx = flag[0] ? (real)0 : vx1, sy = flag[1] ? (real)0 : vx2, sz = flag[2] ? (real)0 : vx3;
                const real feq = feq_bc(drho, cdot(d, vx1, vx2, vx3), cu_sq, w);
                *target = interp_velo(qd, g[d], g[e], feq, omega, cdot(d, sx, sy, sz), w);
                break;
            }
            default:
                break;
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* wall-model (stress) BCs (src/gpu/core/BoundaryConditions/Stress/)         */
/* ------------------------------------------------------------------------ */
/* square root and natural logarithm in the working precision (the float
 * overloads a CUDA build calls on a float) */
#define RSQRT(x) (sizeof(real) == sizeof(float) ? (real)sqrtf((float)(x)) : (real)sqrt((double)(x)))
#define RLOG(x) (sizeof(real) == sizeof(float) ? (real)logf((float)(x)) : (real)log((double)(x)))

/* clip of the wall velocity (iMEM.cuh:131-136): the model's value
 * -3 F forceFactor is formed in double (the literal 3.0 promotes it) and
 * bounded by +-clip, the double min / max ignoring a NaN operand */
static real imem_clip(real clip, real F, real forceFactor)
{
    const double t = -3.0 * (double)F * (double)forceFactor;
    return (real)(clip > -clip ? fmin((double)clip, fmax((double)-clip, t)) : fmax((double)clip, fmin((double)-clip, t)));
}

/* the iMEM wall model of one BC entry (iMEM.cuh:57-137): temporal filters of
 * the velocity at the sampling node kN and at the wall node, the friction
 * velocity from the log law at height samplingOffset + q over z0, the wall
 * shear stress scaled with the wall node's tangential velocity (Schumann-
 * Groetzbach) and the wall velocity that applies the momentum difference.
 * The filter updates mix precisions as the reference writes them: eps * v in
 * the working precision, (1.0 - eps) * mean in double. */
static void imem(uint32_t i, uint32_t kN, const real *nX, const real *nY, const real *nZ, const real *vx,
                 const real *vy, const real *vz, real *vxEl, real *vyEl, real *vzEl, real *vxWMean, real *vyWMean,
                 real *vzWMean, real vxW, real vyW, real vzW, real rho, const int32_t *samplingOffset, real q,
                 real forceFactor, real eps, const real *z0, int hasMonitor, real *uStarMonitor, real wmX, real wmY,
                 real wmZ, real *VX, real *VY, real *VZ)
{
    const real wnx = nX[i], wny = nY[i], wnz = nZ[i];
    real el[3], wm[3];
    el[0] = (real)((double)(eps * vx[kN]) + (1.0 - (double)eps) * (double)vxEl[i]);
    el[1] = (real)((double)(eps * vy[kN]) + (1.0 - (double)eps) * (double)vyEl[i]);
    el[2] = (real)((double)(eps * vz[kN]) + (1.0 - (double)eps) * (double)vzEl[i]);
    vxEl[i] = el[0];
    vyEl[i] = el[1];
    vzEl[i] = el[2];
    wm[0] = (real)((double)(eps * vxW) + (1.0 - (double)eps) * (double)vxWMean[i]);
    wm[1] = (real)((double)(eps * vyW) + (1.0 - (double)eps) * (double)vyWMean[i]);
    wm[2] = (real)((double)(eps * vzW) + (1.0 - (double)eps) * (double)vzWMean[i]);
    vxWMean[i] = wm[0];
    vyWMean[i] = wm[1];
    vzWMean[i] = wm[2];

    /* tangential parts */
    const real dEl = el[0] * wnx + el[1] * wny + el[2] * wnz;
    el[0] -= dEl * wnx;
    el[1] -= dEl * wny;
    el[2] -= dEl * wnz;
    const real magEl = RSQRT(el[0] * el[0] + el[1] * el[1] + el[2] * el[2]);
    const real dWm = wm[0] * wnx + wm[1] * wny + wm[2] * wnz;
    wm[0] -= dWm * wnx;
    wm[1] -= dWm * wny;
    wm[2] -= dWm * wnz;
    const real magWm = RSQRT(wm[0] * wm[0] + wm[1] * wm[1] + wm[2] * wm[2]);
    const real dW = vxW * wnx + vyW * wny + vzW * wnz;
    const real tx = vxW - dW * wnx, ty = vyW - dW * wny, tz = vzW - dW * wnz;

    const real z = (real)samplingOffset[i] + q;
    const real kappa = (real)0.4;
    const real uStar = magEl * kappa / (RLOG(z / z0[i]));
    if (hasMonitor)
        uStarMonitor[i] = uStar;
    const real tauW = uStar * uStar;
    const real A = (real)1.0;
    const real Fwx = (tauW * A) * (tx / magWm);
    const real Fwy = (tauW * A) * (ty / magWm);
    const real Fwz = (tauW * A) * (tz / magWm);
    const real dM = wmX * wnx + wmY * wny + wmZ * wnz;
    const real Fx = Fwx - (wmX - dM * wnx) / rho;
    const real Fy = Fwy - (wmY - dM * wny) / rho;
    const real Fz = Fwz - (wmZ - dM * wnz) / rho;
    const real clip = (real)2.0;
    *VX = imem_clip(clip * el[0], Fx, forceFactor);
    *VY = imem_clip(clip * el[1], Fy, forceFactor);
    *VZ = imem_clip(clip * el[2], Fz, forceFactor);
}

#define BC_STRESS_INTERP 0
#define BC_STRESS_BB 1
#define BC_STRESS_BB_PRESSURE 2

/* wall-model BC over one list, one entry after another:
 *   StressCompressible_Device (StressCompressible.cu:50-762): interpolated
 *     bounce-back with the pressure term (KernelUtilities.h:199-206) and the
 *     relaxation rate om1 / (1 + 3 om1 max(0, nu_t)); the wall velocity's term
 *     divided by 1 + q, force factor 1 + q_B;
 *   StressBounceBackCompressible_Device (StressBounceBackCompressible.cu:50-679):
 *     simple bounce-back, force factor 1;
 *   StressBounceBackPressureCompressible_Device
 *     (StressBounceBackPressureCompressible.cu): simple bounce-back minus w drho.
 * The first pass forms every incoming population of a wall direction and the
 * momentum exchanged with the wall at rest, iMEM turns it into a wall
 * velocity, the second pass writes the incoming populations with the wall
 * velocity's term.  StressCompressible_Device weighs the pressure term of its
 * dPP0 direction with 2/27 (StressCompressible.cu:293); kept.  turbViscosity
 * may be NULL (no turbulence model: the rate is om1). */
void FN(vfo_bc_stress)(int kind, real *dist, uint64_t N, const uint32_t *nx, const uint32_t *ny, const uint32_t *nz,
                       const int32_t *bcNodes, const int32_t *samplingNodes, const real *q, uint32_t nBC, real omega,
                       const real *turbViscosity, const real *vx, const real *vy, const real *vz, const real *normalX,
                       const real *normalY, const real *normalZ, real *vxEl, real *vyEl, real *vzEl, real *vxWMean,
                       real *vyWMean, real *vzWMean, const int32_t *samplingOffset, const real *z0, int hasMonitor,
                       real *uStar, real *Fx, real *Fy, real *Fz, int isEven)
{
    for (uint32_t i = 0; i < nBC; ++i) {
        const locs8 L = list_indices((uint32_t)bcNodes[i], nx, ny, nz);
        real g[27];
        for (int d = 0; d < 27; ++d)
            g[d] = post_value(dist, N, &L, isEven, d);
        real drho, vx1, vx2, vx3;
        bc_macros(g, &drho, &vx1, &vx2, &vx3);
        const real cu_sq = C(3, 2) * (vx1 * vx1 + vx2 * vx2 + vx3 * vx3) * ((real)1 + drho);
        real omTurb = omega;
        if (kind == BC_STRESS_INTERP && turbViscosity) {
            const real nu = turbViscosity[bcNodes[i]];
            omTurb = omega / ((real)1 + (real)3 * omega * (nu > (real)0 ? nu : (real)0));
        }
        const int odd = !isEven;
        real fin[27];
        real wmX = 0, wmY = 0, wmZ = 0;
        for (int j = 0; j < 26; ++j) {
            const int d = QORDER[j];
            const real qd = q[(uint64_t)d * nBC + i];
            if (!(qd >= (real)0 && qd <= (real)1))
                continue;
            const int e = INV[d];
            const real w = weight_of(d);
            if (kind == BC_STRESS_BB) {
                fin[d] = g[d];
            } else if (kind == BC_STRESS_BB_PRESSURE) {
                fin[d] = g[d] - w * drho;
            } else {
                const real feq = feq_bc(drho, cdot(d, vx1, vx2, vx3), cu_sq, w);
                const real wp = d == dPP0 ? C(2, 27) : w;
                fin[d] = interp_noslip(qd, g[d], g[e], feq, omTurb) - wp * drho;
            }
            const real t = g[d] + fin[d];
            if (CX[d] > 0) wmX += t; else if (CX[d] < 0) wmX -= t;
            if (CY[d] > 0) wmY += t; else if (CY[d] < 0) wmY -= t;
            if (CZ[d] > 0) wmZ += t; else if (CZ[d] < 0) wmZ -= t;
        }
        const real qB = q[(uint64_t)d00M * nBC + i];
        const real forceFactor = kind == BC_STRESS_INTERP ? (real)(1.0 + (double)qB) : (real)1.0;
        real VX, VY, VZ;
        imem(i, (uint32_t)samplingNodes[i], normalX, normalY, normalZ, vx, vy, vz, vxEl, vyEl, vzEl, vxWMean, vyWMean,
             vzWMean, vx1, vx2, vx3, (real)1 + drho, samplingOffset, qB, forceFactor, (real)0.001f, z0, hasMonitor, uStar,
             wmX, wmY, wmZ, &VX, &VY, &VZ);
        for (int j = 0; j < 26; ++j) {
            const int d = QORDER[j];
            const real qd = q[(uint64_t)d * nBC + i];
            if (!(qd >= (real)0 && qd <= (real)1))
                continue;
            const int e = INV[d];
            real term = (real)6 * weight_of(d) * cdot(d, VX, VY, VZ);
            if (kind == BC_STRESS_INTERP)
                term = term / ((real)1 + qd);
            dist[(uint64_t)slot_of(e, odd) * N + L.k[loc_of(e)]] = fin[d] - term;
            if (CX[d] > 0) wmX -= term; else if (CX[d] < 0) wmX += term;
            if (CY[d] > 0) wmY -= term; else if (CY[d] < 0) wmY += term;
            if (CZ[d] > 0) wmZ -= term; else if (CZ[d] < 0) wmZ += term;
        }
        if (hasMonitor) {
            Fx[i] = wmX;
            Fy[i] = wmY;
            Fz[i] = wmZ;
        }
    }
}

/* pre-collision non-equilibrium pressure BC, one directional list
 * (PressureNonEquilibriumCompressible.cu:45-311).  direction is the D3Q27 id
 * of the boundary normal (dM00, dP00, d0M0, d0P0, d00M or d00P). */
void FN(vfo_bc_pressure_noneq)(real *dist, uint64_t N, const uint32_t *nx, const uint32_t *ny, const uint32_t *nz,
                               const int32_t *bcNodes, const int32_t *bcNeighbors, const real *rhoBC, uint32_t nBC,
                               int direction, int isEven)
{
    const int axis = CX[direction] != 0 ? 0 : CY[direction] != 0 ? 1 : 2;
    const int sgn = axis == 0 ? CX[direction] : axis == 1 ? CY[direction] : CZ[direction];
    for (uint32_t i = 0; i < nBC; ++i) {
        const locs8 L = list_indices((uint32_t)bcNodes[i], nx, ny, nz);
        const locs8 LN = list_indices((uint32_t)bcNeighbors[i], nx, ny, nz);
        real f[27];
        gather_pre(f, dist, N, &LN, isEven);
        real drho1 = pyramid_density(f);
        const real oneOverRho = (real)1 / (drho1 + (real)1);
        const real vx1 = pyramid_jx(f) * oneOverRho;
        const real vx2 = pyramid_jy(f) * oneOverRho;
        const real vx3 = pyramid_jz(f) * oneOverRho;
        const real cusq = C(3, 2) * (vx1 * vx1 + vx2 * vx2 + vx3 * vx3);
        for (int d = 0; d < 27; ++d) {
            if (d == d000) {
                f[d] -= C(8, 27) * (drho1 - (drho1 + (real)1) * cusq);
            } else {
                const real cu = cdot(d, vx1, vx2, vx3);
                f[d] -= weight_of(d) * (drho1 + (drho1 + (real)1) * ((real)3 * (cu) + C(9, 2) * (cu) * (cu) - cusq));
            }
        }
        drho1 = rhoBC[i];
        for (int d = 0; d < 27; ++d) {
            if (d == d000) {
                f[d] += C(8, 27) * (drho1 - (drho1 + (real)1) * cusq);
            } else {
                const real cu = cdot(d, vx1, vx2, vx3);
                f[d] += weight_of(d) * (drho1 + (drho1 + (real)1) * ((real)3 * (cu) + C(9, 2) * (cu) * (cu) - cusq));
            }
        }
        for (int d = 0; d < 27; ++d) {
            const int c = axis == 0 ? CX[d] : axis == 1 ? CY[d] : CZ[d];
            if (c == sgn)
                continue;
            dist[(uint64_t)slot_of(d, isEven) * N + L.k[loc_of(d)]] = f[d];
        }
    }
}

/* Non-reflecting outflow, one directional list: OutflowNonReflecting_Device
 * (OutflowNonReflecting.cu:50-276) when correction == 0,
 * OutflowNonReflectingPressureCorrection_Device
 * (OutflowNonReflectingPressureCorrection.cu:51-241) otherwise.  For the nine
 * directions whose component along the normal's axis is opposite to the
 * normal, the BC node gets cs f_neighbour + (1 - cs) f_node (minus
 * w_d factor drho_node with the correction), cs = 1 / sqrtf(3) formed from a
 * single-precision square root as in the reference.  Both read the current
 * view and write the other view (:199 / :164).  The corrected form reads the
 * neighbour's populations at the neighbour itself for the directions without
 * a negative component, but at the BC node's shifted locations for the others
 * (its kN_* indices are taken from the BC node, :89-96); that is reproduced. */
void FN(vfo_bc_outflow)(int correction, real *dist, uint64_t N, const uint32_t *nx, const uint32_t *ny,
                        const uint32_t *nz, const int32_t *bcNodes, const int32_t *bcNeighbors, uint32_t nBC,
                        int direction, real factor, int isEven)
{
    const int axis = CX[direction] != 0 ? 0 : CY[direction] != 0 ? 1 : 2;
    const int sgn = axis == 0 ? CX[direction] : axis == 1 ? CY[direction] : CZ[direction];
    const real cs = (real)1 / (real)sqrtf(3.0f);
    for (uint32_t i = 0; i < nBC; ++i) {
        const locs8 L = list_indices((uint32_t)bcNodes[i], nx, ny, nz);
        locs8 LN;
        if (correction) {
            LN = L;
            LN.k[0] = (uint32_t)bcNeighbors[i];
        } else {
            LN = list_indices((uint32_t)bcNeighbors[i], nx, ny, nz);
        }
        real f[27], fN[27];
        gather_pre(f, dist, N, &L, isEven);
        gather_pre(fN, dist, N, &LN, isEven);
        const real rhoCorrection = correction ? factor * pyramid_density(f) : (real)0;
        for (int d = 1; d < 27; ++d) {
            const int c = axis == 0 ? CX[d] : axis == 1 ? CY[d] : CZ[d];
            if (c != -sgn)
                continue;
            real v = fN[d] * cs + ((real)1 - cs) * f[d];
            if (correction)
                v = v - weight_of(d) * rhoCorrection;
            dist[(uint64_t)slot_of(d, !isEven) * N + L.k[loc_of(d)]] = v;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* macroscopic output and reductions                                          */
/* ------------------------------------------------------------------------ */
/* enstrophy of one node (EnstrophyAnalyzer.cu:112-338): 1/2 (drho + 1) |curl u|^2
 * with one-sided reach: the six axis neighbours must be fluid, and each axis
 * uses the widest central difference (order 8, 6, 4 or 2) whose stencil
 * stays on fluid nodes.  Negative steps go through the inverse (-x-y-z)
 * neighbour and two positive steps, as everywhere in the reference. */
#define GEO_FLUID_NODE 19

static uint32_t step_plus(int axis, uint32_t k, const uint32_t *nx, const uint32_t *ny, const uint32_t *nz)
{
    return axis == 0 ? nx[k] : axis == 1 ? ny[k] : nz[k];
}

static uint32_t step_minus(int axis, uint32_t k, const uint32_t *nx, const uint32_t *ny, const uint32_t *nz,
                           const uint32_t *nneg)
{
    const uint32_t w = nneg[k];
    return axis == 0 ? nz[ny[w]] : axis == 1 ? nz[nx[w]] : ny[nx[w]];
}

/* d u / d x_axis with the central difference of the given order (:285-327) */
static real central_difference(const real *u, const uint32_t P[4], const uint32_t M[4], int order)
{
    if (order == 2)
        return (u[P[0]] - u[M[0]]) / (real)2;
    if (order == 4)
        return (((real)8 * u[P[0]] - (real)8 * u[M[0]]) - (u[P[1]] - u[M[1]])) / (real)12;
    if (order == 6)
        return (((real)5 * (real)9) * (u[P[0]] - u[M[0]]) - (real)9 * (u[P[1]] - u[M[1]]) + (u[P[2]] - u[M[2]])) /
               ((real)6 * (real)10);
    return (((real)28 * (real)8) * (u[P[0]] - u[M[0]]) - ((real)7 * (real)8) * (u[P[1]] - u[M[1]]) +
            ((real)8 * (real)4 * C(1, 3)) * (u[P[2]] - u[M[2]]) - (u[P[3]] - u[M[3]])) /
           ((real)7 * (real)10 * (real)4);
}

void FN(vfo_enstrophy_nodes)(const real *rho, const real *vx, const real *vy, const real *vz, uint64_t N,
                             const uint32_t *geo, const uint32_t *nx, const uint32_t *ny, const uint32_t *nz,
                             const uint32_t *nneg, real *out, uint32_t *isFluid)
{
    for (uint64_t kk = 0; kk < N; ++kk) {
        const uint32_t k = (uint32_t)kk;
        out[k] = 0;
        isFluid[k] = 0;
        if (geo[k] != GEO_FLUID_NODE)
            continue;
        uint32_t P[3][4], M[3][4];
        int order[3] = { 8, 8, 8 }, reach = 1;
        for (int a = 0; a < 3; ++a) {
            P[a][0] = step_plus(a, k, nx, ny, nz);
            M[a][0] = step_minus(a, k, nx, ny, nz, nneg);
            if (geo[P[a][0]] != GEO_FLUID_NODE || geo[M[a][0]] != GEO_FLUID_NODE)
                reach = 0;
        }
        if (!reach)
            continue;
        for (int a = 0; a < 3; ++a) {
            for (int i = 1; i < 4; ++i) {
                P[a][i] = step_plus(a, P[a][i - 1], nx, ny, nz);
                M[a][i] = step_minus(a, M[a][i - 1], nx, ny, nz, nneg);
                const int cap = 2 * i; /* a non-fluid node at distance i + 1 caps the order at 2 i */
                if ((geo[P[a][i]] != GEO_FLUID_NODE || geo[M[a][i]] != GEO_FLUID_NODE) && order[a] > cap)
                    order[a] = cap;
            }
        }
        const real dxvy = central_difference(vy, P[0], M[0], order[0]);
        const real dxvz = central_difference(vz, P[0], M[0], order[0]);
        const real dyvx = central_difference(vx, P[1], M[1], order[1]);
        const real dyvz = central_difference(vz, P[1], M[1], order[1]);
        const real dzvx = central_difference(vx, P[2], M[2], order[2]);
        const real dzvy = central_difference(vy, P[2], M[2], order[2]);
        const real wx = dyvz - dzvy, wy = dzvx - dxvz, wz = dxvy - dyvx;
        isFluid[k] = 1;
        out[k] = C(1, 2) * (rho[k] + (real)1) * (wx * wx + wy * wy + wz * wz);
    }
}
/* rho (drho) and velocity of every valid node from its pre-collision view,
 * with the pyramid sums of MacroscopicQuantities.h:117-127 */
void FN(vfo_macroscopic)(const real *dist, uint64_t N, const uint32_t *geo, const uint32_t *nx, const uint32_t *ny,
                         const uint32_t *nz, int isEven, real *rho, real *vx, real *vy, real *vz)
{
    for (uint64_t kk = 0; kk < N; ++kk) {
        const uint32_t k = (uint32_t)kk;
        rho[k] = 0;
        vx[k] = 0;
        vy[k] = 0;
        vz[k] = 0;
        if (geo[k] == GEO_SOLID || geo[k] == GEO_VOID)
            continue;
        locs8 L = list_indices(k, nx, ny, nz);
        real f[27];
        gather_pre(f, dist, N, &L, isEven);
        const real drho = pyramid_density(f);
        const real oneOverRho = (real)1 / (drho + (real)1);
        rho[k] = drho;
        vx[k] = pyramid_jx(f) * oneOverRho;
        vy[k] = pyramid_jy(f) * oneOverRho;
        vz[k] = pyramid_jz(f) * oneOverRho;
    }
}

/* ------------------------------------------------------------------------ */
/* exported primitives for the known-answer tests of the reference's unit     */
/* tests (tests/unit-tests/lbm/ChimeraTests.cpp, MacroscopicQuantitiesTests.cpp, */
/* tests/unit-tests/gpu/core/Utilities/KernelUtilitiesTests.cpp)            */
/* ------------------------------------------------------------------------ */
void FN(vfo_chimera)(int which, real *abc, real vv, real v2, real kinv, real k)
{
    switch (which) {
    case 0: fwd_k(&abc[0], &abc[1], &abc[2], vv, v2, kinv, k); break;
    case 1: bwd_k(&abc[0], &abc[1], &abc[2], vv, v2, kinv, k); break;
    case 2: fwd_0(&abc[0], &abc[1], &abc[2], vv, v2); break;
    default: bwd_0(&abc[0], &abc[1], &abc[2], vv, v2); break;
    }
}

/* out: density, jx, jy, jz (incompressible sums), then the compressible
 * drho, vx, vy, vz of getCompressibleMacroscopicValues */
void FN(vfo_macros)(const real *f, real *out)
{
    out[0] = pyramid_density(f);
    out[1] = pyramid_jx(f);
    out[2] = pyramid_jy(f);
    out[3] = pyramid_jz(f);
    const real oneOverRho = (real)1 / (out[0] + (real)1);
    out[4] = out[0];
    out[5] = out[1] * oneOverRho;
    out[6] = out[2] * oneOverRho;
    out[7] = out[3] * oneOverRho;
}

/* array slot read for direction d in the given parity view */
int FN(vfo_slot)(int d, int isEven) { return slot_of(d, isEven); }
