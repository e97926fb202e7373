"""A plain PyTorch transcription of the single-level time step (TEST
INFRASTRUCTURE: the FP64 autograd reference for the library's hand-written
adjoint).

Every function here restates the oracle's C (oracle/vf_oracle.c) with torch
tensors so that autograd can differentiate it:
  k17()            vfo_k17_collide  (K17CompressibleNavierStokes.h:87-591)
  Step.collision   vfo_collision_k17 (RunCollision.cuh:74-143, twist views
                   KernelUtilities.h:221-379)
  Step.post_bc     vfo_bc_post kinds 0 and 2 (NoSlipInterpolatedCompressible.cu,
                   VelocityInterpolatedCompressible.cu, KernelUtilities.h:171-195)
  Step.pressure    vfo_bc_pressure_noneq (PressureNonEquilibriumCompressible.cu:45-311)
in the order of UpdateGrid27 (UpdateGrid27.cpp:54-96).  Nodes of a BC list are
applied together (every read before any write), as the GPU kernels do.
"""
from __future__ import annotations

import numpy as np
import torch

CX = [0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1]
CY = [0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, -1]
CZ = [0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, 1, 1, 1, -1, -1, -1, -1]
INV = [0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17, 26, 25, 24, 23, 22, 21, 20, 19]
(d000, dP00, dM00, d0P0, d0M0, d00P, d00M, dPP0, dMM0, dPM0, dMP0, dP0P, dM0M, dP0M, dM0P, d0PP, d0MM, d0PM, d0MP,
 dPPP, dMPP, dPMP, dMMP, dPPM, dMPM, dPMM, dMMM) = range(27)
QORDER = [dP00, dM00, d0P0, d0M0, d00P, d00M, dPP0, dMM0, dPM0, dMP0, dP0P, dM0M, dP0M, dM0P, d0PP, d0MM, d0PM, d0MP,
          dPPP, dMMM, dPPM, dMMP, dPMP, dMPM, dPMM, dMPP]


def weight(d):
    n = (CX[d] != 0) + (CY[d] != 0) + (CZ[d] != 0)
    return [8 / 27, 2 / 27, 1 / 54, 1 / 216][n]


def loc(d):
    return (CX[d] < 0) | ((CY[d] < 0) << 1) | ((CZ[d] < 0) << 2)


def slot(d, even):
    return d if even else INV[d]


def cdot(d, ux, uy, uz):
    s = None
    for c, u in ((CX[d], ux), (CY[d], uy), (CZ[d], uz)):
        if c == 0:
            continue
        t = u if c > 0 else -u
        s = t if s is None else s + t
    return 0.0 * ux if s is None else s


def list_indices(k, nx, ny, nz):
    """The eight locations of nodes k (KernelUtilities.h:221-245)."""
    k = np.asarray(k, np.int64)
    L = np.zeros((8, len(k)), np.int64)
    L[0] = k
    L[1] = nx[k]
    L[2] = ny[k]
    L[4] = nz[k]
    L[3] = ny[L[1]]
    L[5] = nz[L[1]]
    L[6] = nz[L[2]]
    L[7] = nz[L[3]]
    return L


# ------------------------------------------------------------------ macros --
def pyramid_density(f):
    t1 = ((f[dPPP] + f[dMMM]) + (f[dMPM] + f[dPMP])) + ((f[dMPP] + f[dPMM]) + (f[dMMP] + f[dPPM]))
    t2 = (((f[d0MP] + f[d0PM]) + (f[d0MM] + f[d0PP])) + ((f[dM0P] + f[dP0M]) + (f[dM0M] + f[dP0P]))) + \
        ((f[dMP0] + f[dPM0]) + (f[dMM0] + f[dPP0]))
    t3 = ((f[dM00] + f[dP00]) + (f[d0M0] + f[d0P0])) + (f[d00M] + f[d00P])
    return ((t1 + t2) + f[d000]) + t3


def pyramid_j(f):
    jx = ((((f[dPPP] - f[dMMM]) + (f[dPMP] - f[dMPM])) + ((f[dPMM] - f[dMPP]) + (f[dPPM] - f[dMMP]))) +
          (((f[dP0M] - f[dM0P]) + (f[dP0P] - f[dM0M])) + ((f[dPM0] - f[dMP0]) + (f[dPP0] - f[dMM0])))) + \
        (f[dP00] - f[dM00])
    jy = ((((f[dPPP] - f[dMMM]) + (f[dMPM] - f[dPMP])) + ((f[dMPP] - f[dPMM]) + (f[dPPM] - f[dMMP]))) +
          (((f[d0PM] - f[d0MP]) + (f[d0PP] - f[d0MM])) + ((f[dMP0] - f[dPM0]) + (f[dPP0] - f[dMM0])))) + \
        (f[d0P0] - f[d0M0])
    jz = ((((f[dPPP] - f[dMMM]) + (f[dPMP] - f[dMPM])) + ((f[dMPP] - f[dPMM]) + (f[dMMP] - f[dPPM]))) +
          (((f[d0MP] - f[d0PM]) + (f[d0PP] - f[d0MM])) + ((f[dM0P] - f[dP0M]) + (f[dP0P] - f[dM0M])))) + \
        (f[d00P] - f[d00M])
    return jx, jy, jz


# ------------------------------------------------------------------ chimera --
def fwd_k(a, b, c, vv, v2, kinv, k):
    m2 = a + c
    m1 = c - a
    m0 = m2 + b
    a_new = m0
    m0 = m0 * kinv + 1.0
    return a_new, (m1 * kinv - m0 * vv) * k, ((m2 - 2.0 * m1 * vv) * kinv + v2 * m0) * k


def bwd_k(a, b, c, vv, v2, kinv, k):
    m0 = (((c - b) * 0.5 + b * vv) * kinv + (a * kinv + 1.0) * (v2 - vv) * 0.5) * k
    m1 = (((a - c) - 2.0 * b * vv) * kinv + (a * kinv + 1.0) * (-v2)) * k
    c_new = (((c + b) * 0.5 + b * vv) * kinv + (a * kinv + 1.0) * (v2 + vv) * 0.5) * k
    return m0, m1, c_new


def fwd_0(a, b, c, vv, v2):
    m1 = (a + c) + b
    m2 = c - a
    return m1, m2 - vv * m1, (c + a) + (v2 * m1 - 2.0 * vv * m2)


def bwd_0(a, b, c, vv, v2):
    ma = (c + a * (v2 - vv)) * 0.5 + b * (vv - 0.5)
    mb = ((a - c) - a * v2) - 2.0 * b * vv
    return ma, mb, (c + a * (v2 + vv)) * 0.5 + b * (vv + 0.5)


FWD_Z = [(dMMM, dMM0, dMMP, 36, 1), (dM0M, dM00, dM0P, 9, 1), (dMPM, dMP0, dMPP, 36, 1), (d0MM, d0M0, d0MP, 9, 1),
         (d00M, d000, d00P, 9, 4), (d0PM, d0P0, d0PP, 9, 1), (dPMM, dPM0, dPMP, 36, 1), (dP0M, dP00, dP0P, 9, 1),
         (dPPM, dPP0, dPPP, 36, 1)]
FWD_Y = [(dMMM, dM0M, dMPM, 6, 1), (dMM0, dM00, dMP0, 0, 0), (dMMP, dM0P, dMPP, 18, 1), (d0MM, d00M, d0PM, 3, 2),
         (d0M0, d000, d0P0, 0, 0), (d0MP, d00P, d0PP, 9, 2), (dPMM, dP0M, dPPM, 6, 1), (dPM0, dP00, dPP0, 0, 0),
         (dPMP, dP0P, dPPP, 18, 1)]
FWD_X = [(dMMM, d0MM, dPMM, 1, 1), (dM0M, d00M, dP0M, 0, 0), (dMPM, d0PM, dPPM, 3, 1), (dMM0, d0M0, dPM0, 0, 0),
         (dM00, d000, dP00, 0, 0), (dMP0, d0P0, dPP0, 0, 0), (dMMP, d0MP, dPMP, 3, 1), (dM0P, d00P, dP0P, 0, 0),
         (dMPP, d0PP, dPPP, -3, 9)]
MSLOT = [[[dMMM, dMM0, dMMP], [dM0M, dM00, dM0P], [dMPM, dMP0, dMPP]],
         [[d0MM, d0M0, d0MP], [d00M, d000, d00P], [d0PM, d0P0, d0PP]],
         [[dPMM, dPM0, dPMP], [dP0M, dP00, dP0P], [dPPM, dPP0, dPPP]]]
BWD_X = [((0, 0, 0), (1, 0, 0), (2, 0, 0), 1, 1), ((0, 1, 0), (1, 1, 0), (2, 1, 0), 0, 0),
         ((0, 2, 0), (1, 2, 0), (2, 2, 0), 3, 1), ((0, 0, 1), (1, 0, 1), (2, 0, 1), 0, 0),
         ((0, 1, 1), (1, 1, 1), (2, 1, 1), 0, 0), ((0, 2, 1), (1, 2, 1), (2, 2, 1), 0, 0),
         ((0, 0, 2), (1, 0, 2), (2, 0, 2), 3, 1), ((0, 1, 2), (1, 1, 2), (2, 1, 2), 0, 0),
         ((0, 2, 2), (1, 2, 2), (2, 2, 2), 9, 1)]
BWD_Y = [((0, 0, 0), (0, 1, 0), (0, 2, 0), 6, 1), ((0, 0, 1), (0, 1, 1), (0, 2, 1), 0, 0),
         ((0, 0, 2), (0, 1, 2), (0, 2, 2), 18, 1), ((1, 0, 0), (1, 1, 0), (1, 2, 0), 3, 2),
         ((1, 0, 1), (1, 1, 1), (1, 2, 1), 0, 0), ((1, 0, 2), (1, 1, 2), (1, 2, 2), 9, 2),
         ((2, 0, 0), (2, 1, 0), (2, 2, 0), 6, 1), ((2, 0, 1), (2, 1, 1), (2, 2, 1), 0, 0),
         ((2, 0, 2), (2, 1, 2), (2, 2, 2), 18, 1)]
BWD_Z = [((0, 0, 0), (0, 0, 1), (0, 0, 2), 36, 1), ((0, 1, 0), (0, 1, 1), (0, 1, 2), 9, 1),
         ((0, 2, 0), (0, 2, 1), (0, 2, 2), 36, 1), ((1, 0, 0), (1, 0, 1), (1, 0, 2), 9, 1),
         ((1, 1, 0), (1, 1, 1), (1, 1, 2), 9, 4), ((1, 2, 0), (1, 2, 1), (1, 2, 2), 9, 1),
         ((2, 0, 0), (2, 0, 1), (2, 0, 2), 36, 1), ((2, 1, 0), (2, 1, 1), (2, 1, 2), 9, 1),
         ((2, 2, 0), (2, 2, 1), (2, 2, 2), 36, 1)]


def sweep_fwd(f, lines, vv, v2):
    for a, b, c, kn, kd in lines:
        if kn == 0:
            f[a], f[b], f[c] = fwd_0(f[a], f[b], f[c], vv, v2)
        elif kn < 0:
            f[a], f[b], f[c] = fwd_k(f[a], f[b], f[c], vv, v2, float(-kn), 1.0 / kd)
        else:
            f[a], f[b], f[c] = fwd_k(f[a], f[b], f[c], vv, v2, kn / kd, kd / kn)


def sweep_bwd(f, lines, vv, v2):
    for ia, ib, ic, kn, kd in lines:
        a, b, c = (MSLOT[i][j][k] for i, j, k in (ia, ib, ic))
        if kn == 0:
            f[a], f[b], f[c] = bwd_0(f[a], f[b], f[c], vv, v2)
        else:
            f[a], f[b], f[c] = bwd_k(f[a], f[b], f[c], vv, v2, kn / kd, kd / kn)


def c222_term(M, oor, drho):
    m111, m200, m020, m002 = M(1, 1, 1), M(2, 0, 0), M(0, 2, 0), M(0, 0, 2)
    m022, m202, m220 = M(0, 2, 2), M(2, 0, 2), M(2, 2, 0)
    m011, m101, m110 = M(0, 1, 1), M(1, 0, 1), M(1, 1, 0)
    m211, m121, m112 = M(2, 1, 1), M(1, 2, 1), M(1, 1, 2)
    m120, m102, m210, m012, m201, m021 = M(1, 2, 0), M(1, 0, 2), M(2, 1, 0), M(0, 1, 2), M(2, 0, 1), M(0, 2, 1)
    return ((-4.0 * m111 * m111 - (m200 * m022 + m020 * m202 + m002 * m220) -
             4.0 * (m011 * m211 + m101 * m121 + m110 * m112) - 2.0 * (m120 * m102 + m210 * m012 + m201 * m021)) * oor +
            (4.0 * (m101 * m101 * m020 + m011 * m011 * m200 + m110 * m110 * m002) + 2.0 * (m200 * m020 * m002) +
             16.0 * m110 * m101 * m011) * oor * oor -
            (1 / 3) * (m022 + m202 + m220) * oor - (1 / 9) * (m200 + m020 + m002) * oor +
            (2.0 * (m101 * m101 + m011 * m011 + m110 * m110) + (m002 * m020 + m002 * m200 + m020 * m200) +
             (1 / 3) * (m002 + m020 + m200)) * oor * oor * (2 / 3) +
            (1 / 27) * ((drho * drho - drho) * oor * oor))


def k17(f, omega, lim, fx, fy, fz):
    """vfo_k17_collide on lists of 27 tensors (returns the post-collision list)."""
    f = list(f)
    drho = pyramid_density(f)
    oor = 1.0 / (drho + 1.0)
    jx, jy, jz = pyramid_j(f)
    vvx = jx * oor + fx
    vvy = jy * oor + fy
    vvz = jz * oor + fz
    vx2, vy2, vz2 = vvx * vvx, vvy * vvy, vvz * vvz
    qlP, qlM, qlD = lim
    sweep_fwd(f, FWD_Z, vvz, vz2)
    sweep_fwd(f, FWD_Y, vvy, vy2)
    sweep_fwd(f, FWD_X, vvx, vx2)

    def M(a, b, c):
        return f[MSLOT[a][b][c]]

    def setM(a, b, c, v):
        f[MSLOT[a][b][c]] = v

    OxyyPxzz = 8.0 * (-2.0 + omega) * (1.0 + 2.0 * omega) / (-8.0 - 14.0 * omega + 7.0 * omega * omega)
    OxyyMxzz = 8.0 * (-2.0 + omega) * (-7.0 + 4.0 * omega) / (56.0 - 50.0 * omega + 9.0 * omega * omega)
    Oxyz = 24.0 * (-2.0 + omega) * (-2.0 - 7.0 * omega + 3.0 * omega * omega) / \
        (48.0 + 152.0 * omega - 130.0 * omega * omega + 29.0 * omega * omega * omega)
    factorA = (4.0 + 2.0 * omega - 3.0 * omega * omega) / (2.0 - 7.0 * omega + 5.0 * omega * omega)
    factorB = (4.0 + 28.0 * omega - 14.0 * omega * omega) / (6.0 - 21.0 * omega + 15.0 * omega * omega)

    # orders 4..6 relax to fixed values with O4 = O5 = O6 = 1; the pre-collision
    # cumulants drop out, so only the moments that the back-transform reads matter
    mxxPyyPzz = M(2, 0, 0) + M(0, 2, 0) + M(0, 0, 2)
    mxxMyy = M(2, 0, 0) - M(0, 2, 0)
    mxxMzz = M(2, 0, 0) - M(0, 0, 2)
    mxxyPyzz = M(2, 1, 0) + M(0, 1, 2)
    mxxyMyzz = M(2, 1, 0) - M(0, 1, 2)
    mxxzPyyz = M(2, 0, 1) + M(0, 2, 1)
    mxxzMyyz = M(2, 0, 1) - M(0, 2, 1)
    mxyyPxzz = M(1, 2, 0) + M(1, 0, 2)
    mxyyMxzz = M(1, 2, 0) - M(1, 0, 2)
    Dxy = -3.0 * omega * M(1, 1, 0)
    Dxz = -3.0 * omega * M(1, 0, 1)
    Dyz = -3.0 * omega * M(0, 1, 1)
    dxux = 0.5 * (-omega) * (mxxMyy + mxxMzz) + 0.5 * (M(0, 0, 0) - mxxPyyPzz)
    dyuy = dxux + omega * 1.5 * mxxMyy
    dzuz = dxux + omega * 1.5 * mxxMzz
    mxxPyyPzz = mxxPyyPzz + (M(0, 0, 0) - mxxPyyPzz) - 3.0 * (1.0 - 0.5) * (vx2 * dxux + vy2 * dyuy + vz2 * dzuz)
    mxxMyy = mxxMyy + omega * (-mxxMyy) - 3.0 * (1.0 + 0.5 * (-omega)) * (vx2 * dxux - vy2 * dyuy)
    mxxMzz = mxxMzz + omega * (-mxxMzz) - 3.0 * (1.0 + 0.5 * (-omega)) * (vx2 * dxux - vz2 * dzuz)
    setM(0, 1, 1, M(0, 1, 1) + omega * (-M(0, 1, 1)))
    setM(1, 0, 1, M(1, 0, 1) + omega * (-M(1, 0, 1)))
    setM(1, 1, 0, M(1, 1, 0) + omega * (-M(1, 1, 0)))

    def limited(x, O, ql):
        w = O + (1.0 - O) * torch.abs(x) / (torch.abs(x) + ql)
        return x + w * (-x)

    setM(1, 1, 1, limited(M(1, 1, 1), Oxyz, qlD))
    mxxyPyzz = limited(mxxyPyzz, OxyyPxzz, qlP)
    mxxyMyzz = limited(mxxyMyzz, OxyyMxzz, qlM)
    mxxzPyyz = limited(mxxzPyyz, OxyyPxzz, qlP)
    mxxzMyyz = limited(mxxzMyyz, OxyyMxzz, qlM)
    mxyyPxzz = limited(mxyyPxzz, OxyyPxzz, qlP)
    mxyyMxzz = limited(mxyyMxzz, OxyyMxzz, qlM)

    setM(2, 0, 0, (1 / 3) * (mxxMyy + mxxMzz + mxxPyyPzz))
    setM(0, 2, 0, (1 / 3) * (-2.0 * mxxMyy + mxxMzz + mxxPyyPzz))
    setM(0, 0, 2, (1 / 3) * (mxxMyy - 2.0 * mxxMzz + mxxPyyPzz))
    setM(2, 1, 0, (mxxyMyzz + mxxyPyzz) * 0.5)
    setM(0, 1, 2, (-mxxyMyzz + mxxyPyzz) * 0.5)
    setM(2, 0, 1, (mxxzMyyz + mxxzPyyz) * 0.5)
    setM(0, 2, 1, (-mxxzMyyz + mxxzPyyz) * 0.5)
    setM(1, 2, 0, (mxyyMxzz + mxyyPxzz) * 0.5)
    setM(1, 0, 2, (-mxyyMxzz + mxyyPxzz) * 0.5)

    tau = 1.0 / omega - 0.5
    cm022 = -tau * (dyuy + dzuz) * (2 / 3) * factorA
    cm202 = -tau * (dxux + dzuz) * (2 / 3) * factorA
    cm220 = -tau * (dyuy + dxux) * (2 / 3) * factorA
    cm112 = -tau * Dxy * (1 / 3) * factorB
    cm121 = -tau * Dxz * (1 / 3) * factorB
    cm211 = -tau * Dyz * (1 / 3) * factorB

    setM(2, 1, 1, cm211 + (1 / 3) * ((3.0 * M(2, 0, 0) + 1.0) * M(0, 1, 1) + 6.0 * M(1, 1, 0) * M(1, 0, 1)) * oor)
    setM(1, 2, 1, cm121 + (1 / 3) * ((3.0 * M(0, 2, 0) + 1.0) * M(1, 0, 1) + 6.0 * M(1, 1, 0) * M(0, 1, 1)) * oor)
    setM(1, 1, 2, cm112 + (1 / 3) * ((3.0 * M(0, 0, 2) + 1.0) * M(1, 1, 0) + 6.0 * M(1, 0, 1) * M(0, 1, 1)) * oor)
    setM(2, 2, 0, cm220 + (((M(2, 0, 0) * M(0, 2, 0) + 2.0 * M(1, 1, 0) * M(1, 1, 0)) * 9.0 +
                            3.0 * (M(2, 0, 0) + M(0, 2, 0))) * oor - (drho * oor)) * (1 / 9))
    setM(2, 0, 2, cm202 + (((M(2, 0, 0) * M(0, 0, 2) + 2.0 * M(1, 0, 1) * M(1, 0, 1)) * 9.0 +
                            3.0 * (M(2, 0, 0) + M(0, 0, 2))) * oor - (drho * oor)) * (1 / 9))
    setM(0, 2, 2, cm022 + (((M(0, 0, 2) * M(0, 2, 0) + 2.0 * M(0, 1, 1) * M(0, 1, 1)) * 9.0 +
                            3.0 * (M(0, 0, 2) + M(0, 2, 0))) * oor - (drho * oor)) * (1 / 9))
    setM(1, 2, 2, (1 / 3) * (3.0 * (M(0, 0, 2) * M(1, 2, 0) + M(0, 2, 0) * M(1, 0, 2) + 4.0 * M(0, 1, 1) * M(1, 1, 1) +
                                    2.0 * (M(1, 0, 1) * M(0, 2, 1) + M(1, 1, 0) * M(0, 1, 2))) +
                             (M(1, 2, 0) + M(1, 0, 2))) * oor)
    setM(2, 1, 2, (1 / 3) * (3.0 * (M(0, 0, 2) * M(2, 1, 0) + M(2, 0, 0) * M(0, 1, 2) + 4.0 * M(1, 0, 1) * M(1, 1, 1) +
                                    2.0 * (M(0, 1, 1) * M(2, 0, 1) + M(1, 1, 0) * M(1, 0, 2))) +
                             (M(2, 1, 0) + M(0, 1, 2))) * oor)
    setM(2, 2, 1, (1 / 3) * (3.0 * (M(2, 0, 0) * M(0, 2, 1) + M(0, 2, 0) * M(2, 0, 1) + 4.0 * M(1, 1, 0) * M(1, 1, 1) +
                                    2.0 * (M(1, 0, 1) * M(1, 2, 0) + M(0, 1, 1) * M(2, 1, 0))) +
                             (M(0, 2, 1) + M(2, 0, 1))) * oor)
    setM(2, 2, 2, -c222_term(M, oor, drho))
    setM(1, 0, 0, -M(1, 0, 0))
    setM(0, 1, 0, -M(0, 1, 0))
    setM(0, 0, 1, -M(0, 0, 1))
    sweep_bwd(f, BWD_X, vvx, vx2)
    sweep_bwd(f, BWD_Y, vvy, vy2)
    sweep_bwd(f, BWD_Z, vvz, vz2)
    return f


# ----------------------------------------------------------- the whole step --
class Step:
    """UpdateGrid27's single-level step on a flat FP64 tensor D[27 N] of one
    grid level (a dict of the builder's arrays)."""

    def __init__(self, g, omega, lim=(0.01, 0.01, 0.01), geometry=True, pressure=True):
        self.g, self.omega, self.lim = g, omega, lim
        self.N = len(g["geo"])
        nb = [g["neighborX"].astype(np.int64), g["neighborY"].astype(np.int64), g["neighborZ"].astype(np.int64)]
        self.Lf = list_indices(g["fluid"], *nb)
        self.lists = [("velocity", 2)] + ([("geometry", 0)] if geometry and len(g["geometry.k"]) else [])
        self.L = {name: list_indices(g[f"{name}.k"], *nb) for name, _ in self.lists}
        self.pressure = pressure and "pressure0.k" in g and len(g["pressure0.k"]) > 0
        if self.pressure:
            self.Lp = list_indices(g["pressure0.k"], *nb)
            self.LpN = list_indices(g["pressure0.kN"], *nb)

    def cells(self, L, d, even):
        return torch.from_numpy(slot(d, even) * self.N + L[loc(d)])

    def collision(self, D, even, fx, fy, fz):
        idx = [self.cells(self.Lf, d, even) for d in range(27)]
        b = k17([D[i] for i in idx], self.omega, self.lim, fx, fy, fz)
        return D.index_put((torch.cat(idx),), torch.cat([b[INV[d]] for d in range(27)]))

    def post_bc(self, D, name, kind, even, U=None):
        g, L = self.g, self.L[name]
        n = L.shape[1]
        # g[d]: post-collision population moving in direction d
        gd = [D[self.cells(L, INV[d], even)] for d in range(27)]
        order = [dPMP, dMPP, dPPP, dMMP, dPMM, dMPM, dPPM, dMMM, d0PM, d0MP, d0PP, d0MM, dP0M, dM0P, dP0P, dM0M, dPM0,
                 dMP0, dPP0, dMM0, d00P, d00M, d0P0, d0M0, dP00, dM00, d000]
        s = gd[order[0]]
        for i in order[1:]:
            s = s + gd[i]
        drho = s
        r1 = 1.0 + s
        vx1 = (((gd[dPMP] - gd[dMPM]) - (gd[dMPP] - gd[dPMM])) + ((gd[dPPP] - gd[dMMM]) - (gd[dMMP] - gd[dPPM])) +
               ((gd[dP0M] - gd[dM0P]) + (gd[dP0P] - gd[dM0M])) + ((gd[dPM0] - gd[dMP0]) + (gd[dPP0] - gd[dMM0])) +
               (gd[dP00] - gd[dM00])) / r1
        vx2 = ((-(gd[dPMP] - gd[dMPM]) + (gd[dMPP] - gd[dPMM])) + ((gd[dPPP] - gd[dMMM]) - (gd[dMMP] - gd[dPPM])) +
               ((gd[d0PM] - gd[d0MP]) + (gd[d0PP] - gd[d0MM])) + (-(gd[dPM0] - gd[dMP0]) + (gd[dPP0] - gd[dMM0])) +
               (gd[d0P0] - gd[d0M0])) / r1
        vx3 = (((gd[dPMP] - gd[dMPM]) + (gd[dMPP] - gd[dPMM])) + ((gd[dPPP] - gd[dMMM]) + (gd[dMMP] - gd[dPPM])) +
               (-(gd[d0PM] - gd[d0MP]) + (gd[d0PP] - gd[d0MM])) + ((gd[dP0P] - gd[dM0M]) - (gd[dP0M] - gd[dM0P])) +
               (gd[d00P] - gd[d00M])) / r1
        cu_sq = 1.5 * (vx1 * vx1 + vx2 * vx2 + vx3 * vx3) * (1.0 + drho)
        q = torch.from_numpy(np.ascontiguousarray(g[f"{name}.q"], dtype=np.float64).reshape(27, n))
        targets, values = [], []
        for d in QORDER:
            active = (q[d] >= 0) & (q[d] <= 1)
            if not bool(active.any()):
                continue
            # the formula on the active entries only (inactive q = -1 would
            # divide by zero, and a zero gradient times inf is NaN)
            sel = torch.nonzero(active).flatten()
            e = INV[d]
            w = weight(d)
            qd = q[d][sel]
            fd, fe, dr = gd[d][sel], gd[e][sel], drho[sel]
            feq = w * (dr + 4.5 * cdot(d, vx1[sel], vx2[sel], vx3[sel]) ** 2 * (1.0 + dr) - cu_sq[sel])
            base = (1.0 - qd) / (1.0 + qd) * (fd - fe + (fd + fe - 2.0 * feq * self.omega) / (1.0 - self.omega)) * 0.5
            if kind == 2:
                v = base + (qd * (fd + fe) - 6.0 * w * cdot(d, U[0][sel], U[1][sel], U[2][sel])) / (1.0 + qd)
            else:
                v = base + (qd * (fd + fe)) / (1.0 + qd)
            targets.append(self.cells(L, e, not even)[sel])
            values.append(v)
        return D.index_put((torch.cat(targets),), torch.cat(values))

    def pressure_bc(self, D, even):
        g = self.g
        direction = int(g["pressure0.dir"][0])
        axis = 0 if CX[direction] else 1 if CY[direction] else 2
        sgn = [CX, CY, CZ][axis][direction]
        f = [D[self.cells(self.LpN, d, even)] for d in range(27)]
        drho1 = pyramid_density(f)
        oor = 1.0 / (drho1 + 1.0)
        jx, jy, jz = pyramid_j(f)
        vx1, vx2, vx3 = jx * oor, jy * oor, jz * oor
        cusq = 1.5 * (vx1 * vx1 + vx2 * vx2 + vx3 * vx3)
        rho = torch.from_numpy(np.asarray(g["pressure0.rho"], np.float64))
        targets, values = [], []
        for d in range(27):
            if [CX, CY, CZ][axis][d] == sgn:
                continue
            if d == d000:
                v = f[d] - (8 / 27) * (drho1 - (drho1 + 1.0) * cusq) + (8 / 27) * (rho - (rho + 1.0) * cusq)
            else:
                cu = cdot(d, vx1, vx2, vx3)
                w = weight(d)
                v = f[d] - w * (drho1 + (drho1 + 1.0) * (3.0 * cu + 4.5 * cu * cu - cusq)) + \
                    w * (rho + (rho + 1.0) * (3.0 * cu + 4.5 * cu * cu - cusq))
            targets.append(self.cells(self.Lp, d, even))
            values.append(v)
        return D.index_put((torch.cat(targets),), torch.cat(values))

    def step(self, D, even, U, force_half):
        D = self.collision(D, even, *force_half)
        for name, kind in self.lists:
            D = self.post_bc(D, name, kind, even, U if kind == 2 else None)
        even = not even
        if self.pressure:
            D = self.pressure_bc(D, even)
        return D, even

    def objective(self, D, even, nodes, wx):
        L = list_indices(nodes, self.g["neighborX"].astype(np.int64), self.g["neighborY"].astype(np.int64),
                         self.g["neighborZ"].astype(np.int64))
        f = [D[self.cells(L, d, even)] for d in range(27)]
        jx, _, _ = pyramid_j(f)
        ux = jx / (pyramid_density(f) + 1.0)
        return (torch.from_numpy(np.asarray(wx, np.float64)) * ux).sum()
