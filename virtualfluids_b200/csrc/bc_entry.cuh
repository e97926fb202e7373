// bc_entry.cuh -- one entry of a post-collision BC list: the arithmetic of
// the post-collision BC kernels (bc.cu, one thread per entry) and of the BC
// epilogue of the planned collision kernels (collision_tiled.cuh), which
// applies the BCs of a tile's wall nodes right after their collision.
//
// Kinds: no-slip interpolated (NoSlipInterpolatedCompressible.cu:44-378),
// no-slip bounce-back (NoSlipBounceBack.cu), velocity interpolated
// (VelocityInterpolatedCompressible.cu:44-418), velocity bounce-back
// (VelocityBounceBack.cu), slip (SlipCompressible.cu:45-550) and velocity
// with pressure (VelocityWithPressureInterpolatedCompressible.cu).  An entry
// reads the post-collision populations of its node through the isEven view
// and writes the bounced-back values into the !isEven view
// (NoSlipInterpolatedCompressible.cu:71,165); it reads all of its values
// before it writes.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/vf_b200.h"
#include "bc_math.cuh"
#include "collision_math.cuh"
#include "d3q27.cuh"
#include "storage.cuh"

namespace vfb
{
// entry i of a list of nBC entries whose node has the locations L; q is the
// list's direction-major q array, Vx / Vy / Vz its velocities (velocity kinds)
template <class S, int KIND, bool EVEN>
__device__ __forceinline__ void bcPostEntry(S* __restrict__ dist, unsigned long long N, typename Storage<S>::R omega,
                                            const Locs& L, const typename Storage<S>::R* __restrict__ q, uint32_t nBC,
                                            uint32_t i, const typename Storage<S>::R* __restrict__ Vx,
                                            const typename Storage<S>::R* __restrict__ Vy,
                                            const typename Storage<S>::R* __restrict__ Vz)
{
    using R = typename Storage<S>::R;
    // post-collision population moving in direction d: slot of inv(d), location of inv(d)
    R g[27];
#pragma unroll
    for (int d = 0; d < 27; ++d)
        g[d] = Storage<S>::load(dist + (unsigned long long)slot<EVEN>(inv(d)) * N + L.k[loc(inv(d))], d);

    R drho = R(0), vx1 = R(0), vx2 = R(0), vx3 = R(0), cuSq = R(0);
    if (KIND == VFB_BC_NOSLIP_INTERPOLATED || KIND == VFB_BC_VELOCITY_INTERPOLATED || KIND == VFB_BC_SLIP ||
        KIND == VFB_BC_VELOCITY_WITH_PRESSURE) {
        bcMacros(g, drho, vx1, vx2, vx3);
        cuSq = R(3) / R(2) * (vx1 * vx1 + vx2 * vx2 + vx3 * vx3) * (R(1) + drho);
    }
    R UX = R(0), UY = R(0), UZ = R(0);
    if (KIND == VFB_BC_VELOCITY_INTERPOLATED || KIND == VFB_BC_VELOCITY_BOUNCE_BACK ||
        KIND == VFB_BC_VELOCITY_WITH_PRESSURE) {
        UX = __ldg(Vx + i);
        UY = __ldg(Vy + i);
        UZ = __ldg(Vz + i);
    }
    // slip: normal components are removed for each axis with an active axis direction
    bool flagX = false, flagY = false, flagZ = false;
    // all q values first, so that their loads are in flight together instead
    // of one per direction behind the branch on the previous one
    R qv[26];
#pragma unroll
    for (int j = 0; j < 26; ++j)
        qv[j] = __ldg(q + (unsigned long long)qOrder(j) * nBC + i);
#pragma unroll
    for (int j = 0; j < 26; ++j) {
        const int d = qOrder(j);
        const R qd = qv[j];
        if (!(qd >= R(0) && qd <= R(1)))
            continue;
        const int e = inv(d);
        S* target = dist + (unsigned long long)slot<!EVEN>(e) * N + L.k[loc(e)];
        const R w = weight<R>(d);
        R value;
        if (KIND == VFB_BC_NOSLIP_BOUNCE_BACK) {
            value = g[d];
        } else if (KIND == VFB_BC_VELOCITY_BOUNCE_BACK) {
            // 6 w (-c_d . U) with 6 w = 4/9, 1/9, 1/36 for face, edge, corner directions
            const R k6 = order(d) == 1 ? R(4) / R(9) : order(d) == 2 ? R(1) / R(9) : R(1) / R(36);
            value = g[d] + k6 * cdot<R>(e, UX, UY, UZ);
        } else if (KIND == VFB_BC_NOSLIP_INTERPOLATED) {
            const R feq = feqBC(drho, cdot<R>(d, vx1, vx2, vx3), cuSq, w);
            value = interpNoSlip(qd, g[d], g[e], feq, omega);
        } else if (KIND == VFB_BC_VELOCITY_INTERPOLATED) {
            const R feq = feqBC(drho, cdot<R>(d, vx1, vx2, vx3), cuSq, w);
            value = interpVelocity(qd, g[d], g[e], feq, omega, cdot<R>(d, UX, UY, UZ), w);
        } else if (KIND == VFB_BC_VELOCITY_WITH_PRESSURE) {
            const R feq = feqBC(drho, cdot<R>(d, vx1, vx2, vx3), cuSq, w);
            value = interpVelocity(qd, g[d], g[e], feq, omega, cdot<R>(d, UX, UY, UZ), w) - w * drho;
        } else {
            if (order(d) == 1) {
                if (cx(d) != 0)
                    flagX = true;
                else if (cy(d) != 0)
                    flagY = true;
                else
                    flagZ = true;
            }
            const R sx = flagX ? R(0) : vx1, sy = flagY ? R(0) : vx2, sz = flagZ ? R(0) : vx3;
            const R feq = feqBC(drho, cdot<R>(d, vx1, vx2, vx3), cuSq, w);
            value = interpVelocity(qd, g[d], g[e], feq, omega, cdot<R>(d, sx, sy, sz), w);
        }
        Storage<S>::store(target, value, d);
    }
}

// The BC epilogue of a planned collision: the post-collision BC lists of a
// level whose entries sit on nodes of the plan's bulk tiles are applied by the
// collision kernel to each such node right after the node's own collision,
// while the node's values are still in L2 (the wall nodes of an x face are a
// stride apart, so a separate BC launch reads a 64-byte DRAM burst per value
// and rewrites partial sectors).  A node qualifies when every active link of
// every one of its entries ends on a node that no collision and no other BC
// entry touches (a boundary stopper or a solid node): then the entry's writes
// reach cells nobody reads before the next step, and its reads are its own
// node's post-collision values, exactly as after a separate launch.  The
// entries of a node run in the schedule's list order.  Descriptor in device
// memory, built by the simulation (vfb_collision_plan_set_bc_epilogue).
constexpr int kMaxFusedLists = 4;
constexpr uint32_t kFusedLast = 1u << 27;     // last record of its node
constexpr uint32_t kFusedEntryMask = kFusedLast - 1;

struct BcEpilogue {
    const uint32_t* nodeRecord; // per node: 1 + index of its first record, 0 if none
    const uint32_t* records;    // (list << 28) | kFusedLast on a node's last record | entry
    int kind[kMaxFusedLists];
    uint32_t n[kMaxFusedLists];
    const void* q[kMaxFusedLists];
    const void* V[kMaxFusedLists][3];
    const uint32_t* locations[kMaxFusedLists];
    double omega;
};

template <class S, bool EVEN>
__device__ __noinline__ void bcEpilogueNode(S* __restrict__ dist, unsigned long long N,
                                            const BcEpilogue* __restrict__ F, uint32_t node)
{
    using R = typename Storage<S>::R;
    const uint32_t first = __ldg(F->nodeRecord + node);
    if (first == 0)
        return;
    const R omega = (R)F->omega;
    for (uint32_t j = first - 1;; ++j) {
        const uint32_t rec = __ldg(F->records + j);
        const int list = (int)(rec >> 28);
        const uint32_t i = rec & kFusedEntryMask;
        const uint32_t n = F->n[list];
        Locs L;
#pragma unroll
        for (int l = 0; l < 8; ++l)
            L.k[l] = __ldg(F->locations[list] + (unsigned long long)l * n + i);
        const R* q = static_cast<const R*>(F->q[list]);
        const R* vx = static_cast<const R*>(F->V[list][0]);
        const R* vy = static_cast<const R*>(F->V[list][1]);
        const R* vz = static_cast<const R*>(F->V[list][2]);
        switch (F->kind[list]) {
        case VFB_BC_NOSLIP_INTERPOLATED:
            bcPostEntry<S, VFB_BC_NOSLIP_INTERPOLATED, EVEN>(dist, N, omega, L, q, n, i, vx, vy, vz);
            break;
        case VFB_BC_NOSLIP_BOUNCE_BACK:
            bcPostEntry<S, VFB_BC_NOSLIP_BOUNCE_BACK, EVEN>(dist, N, omega, L, q, n, i, vx, vy, vz);
            break;
        case VFB_BC_VELOCITY_INTERPOLATED:
            bcPostEntry<S, VFB_BC_VELOCITY_INTERPOLATED, EVEN>(dist, N, omega, L, q, n, i, vx, vy, vz);
            break;
        case VFB_BC_VELOCITY_BOUNCE_BACK:
            bcPostEntry<S, VFB_BC_VELOCITY_BOUNCE_BACK, EVEN>(dist, N, omega, L, q, n, i, vx, vy, vz);
            break;
        case VFB_BC_VELOCITY_WITH_PRESSURE:
            bcPostEntry<S, VFB_BC_VELOCITY_WITH_PRESSURE, EVEN>(dist, N, omega, L, q, n, i, vx, vy, vz);
            break;
        default:
            bcPostEntry<S, VFB_BC_SLIP, EVEN>(dist, N, omega, L, q, n, i, vx, vy, vz);
            break;
        }
        if (rec & kFusedLast)
            break;
    }
}
} // namespace vfb
