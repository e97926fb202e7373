// adjoint.cu -- kernels of the adjoint time step (declarations and the
// conventions in adjoint.cuh).  FP32 and FP64 storage; one thread per node.
//
// Collision.  Forward, node k reads a_d from cell c_d = (slot(d), location
// loc(d)) and writes the post-collision population of direction inv(d) back
// into c_d (KernelUtilities.h:252-281, :350-379).  The map is the identity on
// every other cell, so its adjoint replaces lam at the 27 cells of each fluid
// node by J^T lam: the adjoint of output e sits in cell c_inv(e), the adjoint
// of input d goes to c_d.  J^T is the generated reverse sweep k17Adjoint
// (adjoint_ops.gen.cuh), evaluated at the taped pre-collision values.
//
// Post-collision BCs (interpolated no-slip and velocity, KernelUtilities.h:
// 176-195): node k reads g_d (the post-collision population moving in d) from
// its cells of the current view, computes drho and u by plain sums, and for
// each direction d with 0 <= q_d <= 1 overwrites the cell of inv(d) in the
// other view with
//   v_d = A (g_d - g_e + (g_d + g_e - 2 omega feq_d) / (1 - omega)) / 2
//         + (q (g_d + g_e) - 6 w_d c_d.U) / (1 + q),      A = (1 - q) / (1 + q),
//   feq_d = w_d (drho + 9/2 (c_d.u)^2 (1 + drho) - cuSq),  cuSq = 3/2 |u|^2 (1 + drho)
// (e = inv(d); the no-slip form has U = 0).  The partial derivatives below are
// those of these expressions.
//
// Pressure (PressureNonEquilibriumCompressible.cu:75-309): with the
// neighbour's pre-collision values fN, drho_N and u_N (pyramid sums), the BC
// node's directions d whose normal component differs from the normal's get
//   out_d = fN_d + w_d (rho_BC - drho_N) (1 + 3 c_d.u + 9/2 (c_d.u)^2 - 3/2 |u|^2).
#include <cuda_runtime.h>

#include <cstdlib>

#include "adjoint.cuh"
#include "adjoint_ops.gen.cuh"
#include "capi_common.cuh"
#include "d3q27.cuh"
#include "pdl.cuh"

namespace vfb
{
namespace adjoint
{
namespace
{
constexpr int kThreads = 128;
// resident blocks per SM of the collision adjoint (see collisionAdjointKernel)
constexpr int kAdjointBlocksFP32 = 3;
constexpr int kAdjointBlocksFP64 = 2;

unsigned blocksFor(uint32_t n) { return (n + kThreads - 1) / kThreads; }

template <class R>
__device__ __forceinline__ unsigned long long cell(int slotIndex, unsigned long long N, uint32_t location)
{
    return (unsigned long long)slotIndex * N + location;
}

// sum of v over the block, valid in thread 0
__device__ __forceinline__ double blockSum(double v)
{
    __shared__ double part[kThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads(); // part[] may still be read by a previous call
    if (lane == 0)
        part[warp] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kThreads / 32; ++w)
            s += part[w];
    return s;
}

// the eight locations of fluid-list entry i: from the list's location table
// (eight independent loads) when there is one, else through the neighbour arrays
__device__ __forceinline__ Locs fluidLocations(const uint32_t* __restrict__ table, uint32_t i, uint32_t n,
                                               const uint32_t* __restrict__ fluid, const uint32_t* __restrict__ nX,
                                               const uint32_t* __restrict__ nY, const uint32_t* __restrict__ nZ)
{
    if (table) {
        Locs L;
#pragma unroll
        for (int l = 0; l < 8; ++l)
            L.k[l] = __ldg(table + (unsigned long long)l * n + i);
        return L;
    }
    return listIndices(__ldg(fluid + i), nX, nY, nZ);
}

// the eight locations of BC entry i: from the list's location table when it
// has one, else through the neighbour arrays
__device__ __forceinline__ Locs bcEntryLocations(const uint32_t* __restrict__ table, uint32_t i, uint32_t n,
                                                 const int32_t* __restrict__ bcK, const uint32_t* __restrict__ nX,
                                                 const uint32_t* __restrict__ nY, const uint32_t* __restrict__ nZ)
{
    if (table) {
        Locs L;
#pragma unroll
        for (int l = 0; l < 8; ++l)
            L.k[l] = __ldg(table + (unsigned long long)l * n + i);
        return L;
    }
    return listIndices((uint32_t)__ldg(bcK + i), nX, nY, nZ);
}

// ------------------------------------------------------------- collision --
template <class R, bool EVEN>
__global__ void __launch_bounds__(kThreads)
    tapeCollisionKernel(R* __restrict__ dist, unsigned long long N, const uint32_t* __restrict__ nX,
                        const uint32_t* __restrict__ nY, const uint32_t* __restrict__ nZ,
                        const uint32_t* __restrict__ fluid, const uint32_t* __restrict__ table, uint32_t n,
                        const K17Rates<R> r, R fx, R fy, R fz, R* __restrict__ tape)
{
    gridDependencyWait();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const Locs L = fluidLocations(table, i, n, fluid, nX, nY, nZ);
    R f[27];
#pragma unroll
    for (int d = 0; d < 27; ++d)
        f[d] = dist[cell<R>(slot<EVEN>(d), N, L.k[loc(d)])];
    if (tape) {
#pragma unroll
        for (int d = 0; d < 27; ++d)
            tape[(unsigned long long)d * n + i] = f[d];
    }
    R drho, ux, uy, uz;
    k17Collide<R>(f, r, fx, fy, fz, drho, ux, uy, uz);
#pragma unroll
    for (int d = 0; d < 27; ++d)
        dist[cell<R>(slot<EVEN>(d), N, L.k[loc(d)])] = f[inv(d)];
}

// MINB: resident blocks per SM the register allocation aims at (the reverse
// sweep wants more than 128 registers a thread; fewer registers spill to
// local memory but hide more latency)
template <class R, bool EVEN, int MINB>
__global__ void __launch_bounds__(kThreads, MINB)
    collisionAdjointKernel(R* __restrict__ lam, unsigned long long N, const uint32_t* __restrict__ nX,
                           const uint32_t* __restrict__ nY, const uint32_t* __restrict__ nZ,
                           const uint32_t* __restrict__ fluid, const uint32_t* __restrict__ table, uint32_t n,
                           const K17Rates<R> r, R fx, R fy, R fz, const R* __restrict__ tape,
                           double* __restrict__ partials)
{
    gridDependencyWait();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double gx = 0.0, gy = 0.0, gz = 0.0;
    if (i < n) {
        const Locs L = fluidLocations(table, i, n, fluid, nX, nY, nZ);
        R a[27], l[27];
#pragma unroll
        for (int d = 0; d < 27; ++d)
            a[d] = tape[(unsigned long long)d * n + i];
#pragma unroll
        for (int d = 0; d < 27; ++d)
            l[inv(d)] = lam[cell<R>(slot<EVEN>(d), N, L.k[loc(d)])];
        R gfx, gfy, gfz;
        k17Adjoint<R>(a, l, r, fx, fy, fz, gfx, gfy, gfz);
#pragma unroll
        for (int d = 0; d < 27; ++d)
            lam[cell<R>(slot<EVEN>(d), N, L.k[loc(d)])] = l[d];
        gx = (double)gfx;
        gy = (double)gfy;
        gz = (double)gfz;
    }
    gx = blockSum(gx);
    gy = blockSum(gy);
    gz = blockSum(gz);
    // accumulated over the steps of a backward pass, each block in step order
    if (threadIdx.x == 0) {
        partials[3 * blockIdx.x + 0] += gx;
        partials[3 * blockIdx.x + 1] += gy;
        partials[3 * blockIdx.x + 2] += gz;
    }
}

// --------------------------------------------------- post-collision BCs --
// one entry of a forward post-collision list
template <class R, int KIND, bool EVEN>
__device__ __forceinline__ void postBCEntry(R* __restrict__ dist, const BcLattice<R>& lat,
                                            const int32_t* __restrict__ bcK, const uint32_t* __restrict__ table,
                                            const R* __restrict__ q, uint32_t n, const R* __restrict__ Vx,
                                            const R* __restrict__ Vy, const R* __restrict__ Vz, R* __restrict__ rec,
                                            uint32_t i)
{
    const unsigned long long N = lat.N;
    const Locs L = bcEntryLocations(table, i, n, bcK, lat.nX, lat.nY, lat.nZ);
    R g[27];
#pragma unroll
    for (int d = 0; d < 27; ++d)
        g[d] = dist[cell<R>(slot<EVEN>(inv(d)), N, L.k[loc(inv(d))])];
    if (rec) {
#pragma unroll
        for (int d = 0; d < 27; ++d)
            rec[(unsigned long long)d * n + i] = g[d];
    }
    R drho, vx1, vx2, vx3;
    bcMacros(g, drho, vx1, vx2, vx3);
    const R cuSq = R(3) / R(2) * (vx1 * vx1 + vx2 * vx2 + vx3 * vx3) * (R(1) + drho);
    R UX = R(0), UY = R(0), UZ = R(0);
    if (KIND == VFB_BC_VELOCITY_INTERPOLATED) {
        UX = __ldg(Vx + i);
        UY = __ldg(Vy + i);
        UZ = __ldg(Vz + i);
    }
    // all q values first: loads issued together, not one per loop iteration
    R qv[26];
#pragma unroll
    for (int j = 0; j < 26; ++j)
        qv[j] = __ldg(q + (unsigned long long)qOrder(j) * n + i);
#pragma unroll
    for (int j = 0; j < 26; ++j) {
        const int d = qOrder(j);
        const R qd = qv[j];
        if (!(qd >= R(0) && qd <= R(1)))
            continue;
        const int e = inv(d);
        const R w = weight<R>(d);
        const R feq = feqBC(drho, cdot<R>(d, vx1, vx2, vx3), cuSq, w);
        const R value = KIND == VFB_BC_VELOCITY_INTERPOLATED
                            ? interpVelocity(qd, g[d], g[e], feq, lat.omega, cdot<R>(d, UX, UY, UZ), w)
                            : interpNoSlip(qd, g[d], g[e], feq, lat.omega);
        dist[cell<R>(slot<!EVEN>(e), N, L.k[loc(e)])] = value;
    }
}

template <class R, int KIND, bool EVEN>
__global__ void __launch_bounds__(kThreads)
    postBCKernel(R* __restrict__ dist, const BcLattice<R> lat, const int32_t* __restrict__ bcK,
                 const uint32_t* __restrict__ table,
                 const R* __restrict__ q, uint32_t n, const R* __restrict__ Vx, const R* __restrict__ Vy,
                 const R* __restrict__ Vz, R* __restrict__ rec)
{
    gridDependencyWait();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        postBCEntry<R, KIND, EVEN>(dist, lat, bcK, table, q, n, Vx, Vy, Vz, rec, i);
}

template <class R, bool EVEN>
__device__ __forceinline__ void postGatherEntry(R* __restrict__ lam, const BcLattice<R>& lat,
                                                const int32_t* __restrict__ bcK, const uint32_t* __restrict__ table,
                                                const R* __restrict__ q, uint32_t n, R* __restrict__ tmp, uint32_t i)
{
    const Locs L = bcEntryLocations(table, i, n, bcK, lat.nX, lat.nY, lat.nZ);
    // all q values first: loads issued together, not one per loop iteration
    R qv[26];
#pragma unroll
    for (int j = 0; j < 26; ++j)
        qv[j] = __ldg(q + (unsigned long long)qOrder(j) * n + i);
#pragma unroll
    for (int j = 0; j < 26; ++j) {
        const int d = qOrder(j);
        const R qd = qv[j];
        if (!(qd >= R(0) && qd <= R(1)))
            continue;
        const int e = inv(d);
        R* target = lam + cell<R>(slot<!EVEN>(e), lat.N, L.k[loc(e)]);
        tmp[(unsigned long long)d * n + i] = *target;
        *target = R(0);
    }
}

template <class R, bool EVEN>
__global__ void __launch_bounds__(kThreads)
    postGatherKernel(R* __restrict__ lam, const BcLattice<R> lat, const int32_t* __restrict__ bcK,
                     const uint32_t* __restrict__ table, const R* __restrict__ q, uint32_t n, R* __restrict__ tmp)
{
    gridDependencyWait();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        postGatherEntry<R, EVEN>(lam, lat, bcK, table, q, n, tmp, i);
}

template <class R, int KIND, bool EVEN>
__device__ __forceinline__ void postScatterEntry(R* __restrict__ lam, const BcLattice<R>& lat,
                                                 const int32_t* __restrict__ bcK, const uint32_t* __restrict__ table,
                                                 const R* __restrict__ q, uint32_t n, const R* __restrict__ rec,
                                                 const R* __restrict__ tmp, double* __restrict__ gV, uint32_t i)
{
    const Locs L = bcEntryLocations(table, i, n, bcK, lat.nX, lat.nY, lat.nZ);
    R g[27], gg[27];
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        g[d] = rec[(unsigned long long)d * n + i];
        gg[d] = R(0);
    }
    R drho, vx1, vx2, vx3;
    bcMacros(g, drho, vx1, vx2, vx3);
    const R rho = R(1) + drho;
    const R u2 = vx1 * vx1 + vx2 * vx2 + vx3 * vx3;
    const R omega = lat.omega;
    const R c1 = R(1) / (R(1) - omega);
    R gdrho = R(0), gux = R(0), guy = R(0), guz = R(0), gcuSq = R(0);
    R gUx = R(0), gUy = R(0), gUz = R(0);
    // all q values first: loads issued together, not one per loop iteration
    R qv[26];
#pragma unroll
    for (int j = 0; j < 26; ++j)
        qv[j] = __ldg(q + (unsigned long long)qOrder(j) * n + i);
#pragma unroll
    for (int j = 0; j < 26; ++j) {
        const int d = qOrder(j);
        const R qd = qv[j];
        if (!(qd >= R(0) && qd <= R(1)))
            continue;
        const int e = inv(d);
        const R t = tmp[(unsigned long long)d * n + i];
        const R w = weight<R>(d);
        const R A = (R(1) - qd) / (R(1) + qd);
        const R b = qd / (R(1) + qd);
        gg[d] += t * (A * R(0.5) * (R(1) + c1) + b);
        gg[e] += t * (A * R(0.5) * (c1 - R(1)) + b);
        const R gfeq = -t * A * omega * c1;
        const R vel = cdot<R>(d, vx1, vx2, vx3);
        gdrho += gfeq * w * (R(1) + R(4.5) * vel * vel);
        const R gvel = gfeq * w * R(9) * vel * rho;
        gux += gvel * R(cx(d));
        guy += gvel * R(cy(d));
        guz += gvel * R(cz(d));
        gcuSq -= gfeq * w;
        if (KIND == VFB_BC_VELOCITY_INTERPOLATED) {
            const R gU = -t * R(6) * w / (R(1) + qd);
            gUx += gU * R(cx(d));
            gUy += gU * R(cy(d));
            gUz += gU * R(cz(d));
        }
    }
    gdrho += gcuSq * R(1.5) * u2;
    gux += gcuSq * R(3) * vx1 * rho;
    guy += gcuSq * R(3) * vx2 * rho;
    guz += gcuSq * R(3) * vx3 * rho;
    const R oneOverRho = R(1) / rho;
#pragma unroll
    for (int k = 0; k < 27; ++k) {
        const R v = gg[k] + gdrho +
                    (gux * (R(cx(k)) - vx1) + guy * (R(cy(k)) - vx2) + guz * (R(cz(k)) - vx3)) * oneOverRho;
        // atomic: a node can appear in a list more than once (an edge node of
        // two walls, with the directions of each wall), and all its entries
        // add into the same cells
        atomicAdd(lam + cell<R>(slot<EVEN>(inv(k)), lat.N, L.k[loc(inv(k))]), v);
    }
    if (KIND == VFB_BC_VELOCITY_INTERPOLATED && gV) {
        gV[i] += (double)gUx;
        gV[(unsigned long long)n + i] += (double)gUy;
        gV[2ull * n + i] += (double)gUz;
    }
}

template <class R, int KIND, bool EVEN>
__global__ void __launch_bounds__(kThreads)
    postScatterKernel(R* __restrict__ lam, const BcLattice<R> lat, const int32_t* __restrict__ bcK,
                      const uint32_t* __restrict__ table, const R* __restrict__ q, uint32_t n,
                      const R* __restrict__ rec, const R* __restrict__ tmp, double* __restrict__ gV)
{
    gridDependencyWait();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        postScatterEntry<R, KIND, EVEN>(lam, lat, bcK, table, q, n, rec, tmp, gV, i);
}

// ------------------------------------------ post-collision lists together --
// One launch over several lists: block b serves the last list whose first
// block is <= b.  Valid when no list writes a cell another list reads or
// writes (the caller checks this once, sim_adjoint.cu), so the lists' order
// within a step does not matter.
template <class R>
__device__ __forceinline__ const PostList<R>& listOf(const PostLists<R>& P, uint32_t& i)
{
    int l = 0;
#pragma unroll
    for (int j = 1; j < kMaxPostLists; ++j)
        if (j < P.count && blockIdx.x >= P.firstBlock[j])
            l = j;
    i = (blockIdx.x - P.firstBlock[l]) * kThreads + threadIdx.x;
    return P.list[l];
}

template <class R, bool EVEN>
__global__ void __launch_bounds__(kThreads) postBCListsKernel(R* __restrict__ dist, const BcLattice<R> lat,
                                                              const PostLists<R> P)
{
    gridDependencyWait();
    uint32_t i;
    const PostList<R>& L = listOf(P, i);
    if (i >= L.n)
        return;
    if (L.kind == VFB_BC_VELOCITY_INTERPOLATED)
        postBCEntry<R, VFB_BC_VELOCITY_INTERPOLATED, EVEN>(dist, lat, L.k, L.table, L.q, L.n, L.Vx, L.Vy, L.Vz,
                                                           L.rec, i);
    else
        postBCEntry<R, VFB_BC_NOSLIP_INTERPOLATED, EVEN>(dist, lat, L.k, L.table, L.q, L.n, L.Vx, L.Vy, L.Vz, L.rec,
                                                         i);
}

template <class R, bool EVEN>
__global__ void __launch_bounds__(kThreads) postGatherListsKernel(R* __restrict__ lam, const BcLattice<R> lat,
                                                                  const PostLists<R> P)
{
    gridDependencyWait();
    uint32_t i;
    const PostList<R>& L = listOf(P, i);
    if (i < L.n)
        postGatherEntry<R, EVEN>(lam, lat, L.k, L.table, L.q, L.n, L.tmp, i);
}

template <class R, bool EVEN>
__global__ void __launch_bounds__(kThreads) postScatterListsKernel(R* __restrict__ lam, const BcLattice<R> lat,
                                                                   const PostLists<R> P)
{
    gridDependencyWait();
    uint32_t i;
    const PostList<R>& L = listOf(P, i);
    if (i >= L.n)
        return;
    if (L.kind == VFB_BC_VELOCITY_INTERPOLATED)
        postScatterEntry<R, VFB_BC_VELOCITY_INTERPOLATED, EVEN>(lam, lat, L.k, L.table, L.q, L.n, L.rec, L.tmp,
                                                                L.gV, i);
    else
        postScatterEntry<R, VFB_BC_NOSLIP_INTERPOLATED, EVEN>(lam, lat, L.k, L.table, L.q, L.n, L.rec, L.tmp,
                                                              nullptr, i);
}

// --------------------------------------------------------------- pressure --
template <class R, bool EVEN>
__global__ void __launch_bounds__(kThreads)
    pressureKernel(R* __restrict__ dist, const BcLattice<R> lat, const int32_t* __restrict__ bcK,
                   const int32_t* __restrict__ bcKN, const R* __restrict__ rhoBC, uint32_t n, int axis, int sgn,
                   R* __restrict__ rec)
{
    gridDependencyWait();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const unsigned long long N = lat.N;
    const Locs L = listIndices((uint32_t)__ldg(bcK + i), lat.nX, lat.nY, lat.nZ);
    const Locs LN = listIndices((uint32_t)__ldg(bcKN + i), lat.nX, lat.nY, lat.nZ);
    R f[27];
#pragma unroll
    for (int d = 0; d < 27; ++d)
        f[d] = dist[cell<R>(slot<EVEN>(d), N, LN.k[loc(d)])];
    if (rec) {
#pragma unroll
        for (int d = 0; d < 27; ++d)
            rec[(unsigned long long)d * n + i] = f[d];
    }
    // the arithmetic of bcPressureKernel (bc.cu), operation for operation
    R drho1 = pyramidDensity(f);
    const R oneOverRho = R(1) / (drho1 + R(1));
    const R vx1 = pyramidJx(f) * oneOverRho;
    const R vx2 = pyramidJy(f) * oneOverRho;
    const R vx3 = pyramidJz(f) * oneOverRho;
    const R cusq = R(3) / R(2) * (vx1 * vx1 + vx2 * vx2 + vx3 * vx3);
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        if (d == d000) {
            f[d] -= R(8) / R(27) * (drho1 - (drho1 + R(1)) * cusq);
        } else {
            const R cu = cdot<R>(d, vx1, vx2, vx3);
            f[d] -= weight<R>(d) * (drho1 + (drho1 + R(1)) * (R(3) * cu + R(9) / R(2) * cu * cu - cusq));
        }
    }
    drho1 = __ldg(rhoBC + i);
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        if (d == d000) {
            f[d] += R(8) / R(27) * (drho1 - (drho1 + R(1)) * cusq);
        } else {
            const R cu = cdot<R>(d, vx1, vx2, vx3);
            f[d] += weight<R>(d) * (drho1 + (drho1 + R(1)) * (R(3) * cu + R(9) / R(2) * cu * cu - cusq));
        }
    }
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        const int c = axis == 0 ? cx(d) : axis == 1 ? cy(d) : cz(d);
        if (c == sgn)
            continue;
        dist[cell<R>(slot<EVEN>(d), N, L.k[loc(d)])] = f[d];
    }
}

template <class R, bool EVEN>
__global__ void __launch_bounds__(kThreads)
    pressureGatherKernel(R* __restrict__ lam, const BcLattice<R> lat, const int32_t* __restrict__ bcK, uint32_t n,
                         int axis, int sgn, R* __restrict__ tmp)
{
    gridDependencyWait();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const Locs L = listIndices((uint32_t)__ldg(bcK + i), lat.nX, lat.nY, lat.nZ);
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        const int c = axis == 0 ? cx(d) : axis == 1 ? cy(d) : cz(d);
        if (c == sgn)
            continue;
        R* target = lam + cell<R>(slot<EVEN>(d), lat.N, L.k[loc(d)]);
        tmp[(unsigned long long)d * n + i] = *target;
        *target = R(0);
    }
}

template <class R, bool EVEN>
__global__ void __launch_bounds__(kThreads)
    pressureScatterKernel(R* __restrict__ lam, const BcLattice<R> lat, const int32_t* __restrict__ bcKN,
                          const R* __restrict__ rhoBC, uint32_t n, int axis, int sgn, const R* __restrict__ rec,
                          const R* __restrict__ tmp)
{
    gridDependencyWait();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const Locs LN = listIndices((uint32_t)__ldg(bcKN + i), lat.nX, lat.nY, lat.nZ);
    R f[27], gf[27];
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        f[d] = rec[(unsigned long long)d * n + i];
        gf[d] = R(0);
    }
    const R drho = pyramidDensity(f);
    const R oneOverRho = R(1) / (drho + R(1));
    const R ux = pyramidJx(f) * oneOverRho, uy = pyramidJy(f) * oneOverRho, uz = pyramidJz(f) * oneOverRho;
    const R cusq = R(1.5) * (ux * ux + uy * uy + uz * uz);
    const R dr = __ldg(rhoBC + i) - drho;
    R gdrho = R(0), gux = R(0), guy = R(0), guz = R(0);
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        const int c = axis == 0 ? cx(d) : axis == 1 ? cy(d) : cz(d);
        if (c == sgn)
            continue;
        const R t = tmp[(unsigned long long)d * n + i];
        const R w = weight<R>(d);
        const R cu = cdot<R>(d, ux, uy, uz);
        gf[d] += t;
        gdrho -= t * w * (R(1) + R(3) * cu + R(4.5) * cu * cu - cusq);
        const R coef = t * w * dr;
        const R s = R(3) + R(9) * cu;
        gux += coef * (s * R(cx(d)) - R(3) * ux);
        guy += coef * (s * R(cy(d)) - R(3) * uy);
        guz += coef * (s * R(cz(d)) - R(3) * uz);
    }
#pragma unroll
    for (int k = 0; k < 27; ++k) {
        const R v = gf[k] + gdrho + (gux * (R(cx(k)) - ux) + guy * (R(cy(k)) - uy) + guz * (R(cz(k)) - uz)) * oneOverRho;
        atomicAdd(lam + cell<R>(slot<EVEN>(k), lat.N, LN.k[loc(k)]), v);
    }
}

// -------------------------------------------------------------- objective --
template <class R, bool EVEN>
__global__ void __launch_bounds__(kThreads)
    objectiveKernel(const R* __restrict__ dist, unsigned long long N, const uint32_t* __restrict__ nX,
                    const uint32_t* __restrict__ nY, const uint32_t* __restrict__ nZ,
                    const uint32_t* __restrict__ nodes, const double* __restrict__ wx, const double* __restrict__ wy,
                    const double* __restrict__ wz, uint32_t n, double* __restrict__ partials, R* __restrict__ lam,
                    double seed)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double val = 0.0;
    if (i < n) {
        const Locs L = listIndices(__ldg(nodes + i), nX, nY, nZ);
        R f[27];
#pragma unroll
        for (int d = 0; d < 27; ++d)
            f[d] = dist[cell<R>(slot<EVEN>(d), N, L.k[loc(d)])];
        const R oneOverRho = R(1) / (pyramidDensity(f) + R(1));
        const R ux = pyramidJx(f) * oneOverRho, uy = pyramidJy(f) * oneOverRho, uz = pyramidJz(f) * oneOverRho;
        const double ax = wx[i], ay = wy[i], az = wz[i];
        val = ax * (double)ux + ay * (double)uy + az * (double)uz;
        if (lam) {
#pragma unroll
            for (int d = 0; d < 27; ++d) {
                const double g = (ax * ((double)cx(d) - (double)ux) + ay * ((double)cy(d) - (double)uy) +
                                  az * ((double)cz(d) - (double)uz)) *
                                 (double)oneOverRho * seed;
                lam[cell<R>(slot<EVEN>(d), N, L.k[loc(d)])] += (R)g;
            }
        }
    }
    val = blockSum(val);
    if (threadIdx.x == 0)
        partials[blockIdx.x] = val;
}

// one block per component: each thread sums a fixed strided subset, then a
// fixed-shape tree (the same order every call)
constexpr int kReduceThreads = 256;
__global__ void __launch_bounds__(kReduceThreads)
    reduceKernel(const double* __restrict__ partials, unsigned blocks, int width, double* acc, double scale)
{
    __shared__ double part[kReduceThreads];
    const int c = blockIdx.x;
    double s = 0.0;
    for (unsigned b = threadIdx.x; b < blocks; b += kReduceThreads)
        s += partials[(unsigned long long)width * b + c];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int h = kReduceThreads / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h)
            part[threadIdx.x] += part[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        acc[c] += scale * part[0];
}

int axisOf(int direction, int& axis, int& sgn)
{
    if (direction < dP00 || direction > d00M)
        return setError(VFB_ERR_INVALID_ARGUMENT, "direction %d is not an axis direction (1..6)", direction);
    axis = cx(direction) != 0 ? 0 : cy(direction) != 0 ? 1 : 2;
    sgn = axis == 0 ? cx(direction) : axis == 1 ? cy(direction) : cz(direction);
    return VFB_OK;
}
} // namespace

unsigned collisionBlocks(uint32_t nFluid) { return blocksFor(nFluid); }
unsigned objectiveBlocks(uint32_t n) { return blocksFor(n); }

template <class R>
int collision(R* dist, unsigned long long N, const uint32_t* nX, const uint32_t* nY, const uint32_t* nZ,
              const uint32_t* fluid, const uint32_t* loc, uint32_t nFluid, const K17Rates<R>& rates, R fx, R fy, R fz,
              bool even, R* tape, cudaStream_t s)
{
    if (nFluid == 0)
        return VFB_OK;
    const unsigned b = blocksFor(nFluid);
    if (even)
        launchDependent(tapeCollisionKernel<R, true>, b, kThreads, 0, s, dist, N, nX, nY, nZ, fluid, loc, nFluid,
                        rates, fx, fy, fz, tape);
    else
        launchDependent(tapeCollisionKernel<R, false>, b, kThreads, 0, s, dist, N, nX, nY, nZ, fluid, loc, nFluid,
                        rates, fx, fy, fz, tape);
    return checkLaunch("adjoint forward collision");
}

template <class R, int MINB>
void launchCollisionAdjoint(bool even, unsigned b, cudaStream_t s, R* lam, unsigned long long N, const uint32_t* nX,
                            const uint32_t* nY, const uint32_t* nZ, const uint32_t* fluid, const uint32_t* loc,
                            uint32_t nFluid, const K17Rates<R>& rates, R fx, R fy, R fz, const R* tape,
                            double* partials)
{
    if (even)
        launchDependent(collisionAdjointKernel<R, true, MINB>, b, kThreads, 0, s, lam, N, nX, nY, nZ, fluid, loc,
                        nFluid, rates, fx, fy, fz, tape, partials);
    else
        launchDependent(collisionAdjointKernel<R, false, MINB>, b, kThreads, 0, s, lam, N, nX, nY, nZ, fluid, loc,
                        nFluid, rates, fx, fy, fz, tape, partials);
}

static int collisionAdjointOccupancy(bool dbl)
{
    // measured defaults (FP32: 3 blocks of 128 threads per SM; FP64: 2); the
    // environment variable VFB_ADJOINT_BLOCKS (2, 3 or 4) overrides them for tuning
    static const int env = [] {
        const char* e = std::getenv("VFB_ADJOINT_BLOCKS");
        const int v = e ? std::atoi(e) : 0;
        return v >= 2 && v <= 4 ? v : 0;
    }();
    if (env)
        return env;
    return dbl ? kAdjointBlocksFP64 : kAdjointBlocksFP32;
}

template <class R>
int collisionAdjoint(R* lam, unsigned long long N, const uint32_t* nX, const uint32_t* nY, const uint32_t* nZ,
                     const uint32_t* fluid, const uint32_t* loc, uint32_t nFluid, const K17Rates<R>& rates, R fx,
                     R fy, R fz, bool even, const R* tape, double* partials, cudaStream_t s)
{
    if (nFluid == 0)
        return VFB_OK;
    const unsigned b = blocksFor(nFluid);
    switch (collisionAdjointOccupancy(sizeof(R) == 8)) {
    case 2: launchCollisionAdjoint<R, 2>(even, b, s, lam, N, nX, nY, nZ, fluid, loc, nFluid, rates, fx, fy, fz, tape,
                                         partials); break;
    case 3: launchCollisionAdjoint<R, 3>(even, b, s, lam, N, nX, nY, nZ, fluid, loc, nFluid, rates, fx, fy, fz, tape,
                                         partials); break;
    default: launchCollisionAdjoint<R, 4>(even, b, s, lam, N, nX, nY, nZ, fluid, loc, nFluid, rates, fx, fy, fz, tape,
                                          partials); break;
    }
    return checkLaunch("collision adjoint");
}

template <class R, int KIND, bool EVEN>
void launchPostBC(unsigned b, cudaStream_t s, R* dist, const BcLattice<R>& lat, const int32_t* k,
                  const uint32_t* table, const R* q, uint32_t n, const R* Vx, const R* Vy, const R* Vz, R* rec)
{
    launchDependent(postBCKernel<R, KIND, EVEN>, b, kThreads, 0, s, dist, lat, k, table, q, n, Vx, Vy, Vz, rec);
}

template <class R>
int postBC(int kind, R* dist, const BcLattice<R>& lat, const int32_t* k, const uint32_t* table, const R* q, uint32_t n,
           const R* Vx, const R* Vy, const R* Vz, bool even, R* rec, cudaStream_t s)
{
    if (n == 0)
        return VFB_OK;
    const unsigned b = blocksFor(n);
    constexpr int V = VFB_BC_VELOCITY_INTERPOLATED, NS = VFB_BC_NOSLIP_INTERPOLATED;
    if (kind == V)
        (even ? launchPostBC<R, V, true> : launchPostBC<R, V, false>)(b, s, dist, lat, k, table, q, n, Vx, Vy, Vz, rec);
    else if (kind == NS)
        (even ? launchPostBC<R, NS, true> : launchPostBC<R, NS, false>)(b, s, dist, lat, k, table, q, n, Vx, Vy, Vz,
                                                                       rec);
    else
        return setError(VFB_ERR_INVALID_ARGUMENT, "BC kind %d has no adjoint", kind);
    return checkLaunch("adjoint forward BC");
}

template <class R, int KIND, bool EVEN>
void launchPostScatter(unsigned b, cudaStream_t s, R* lam, const BcLattice<R>& lat, const int32_t* k,
                       const uint32_t* table, const R* q, uint32_t n, const R* rec, const R* tmp, double* gV)
{
    launchDependent(postScatterKernel<R, KIND, EVEN>, b, kThreads, 0, s, lam, lat, k, table, q, n, rec, tmp, gV);
}

template <class R>
int postBCAdjoint(int kind, R* lam, const BcLattice<R>& lat, const int32_t* k, const uint32_t* table, const R* q,
                  uint32_t n, const R* Vx, const R* Vy, const R* Vz, bool even, const R* rec, R* tmp, double* gV,
                  cudaStream_t s)
{
    (void)Vx;
    (void)Vy;
    (void)Vz;
    if (n == 0)
        return VFB_OK;
    if (kind != VFB_BC_VELOCITY_INTERPOLATED && kind != VFB_BC_NOSLIP_INTERPOLATED)
        return setError(VFB_ERR_INVALID_ARGUMENT, "BC kind %d has no adjoint", kind);
    const unsigned b = blocksFor(n);
    if (even)
        launchDependent(postGatherKernel<R, true>, b, kThreads, 0, s, lam, lat, k, table, q, n, tmp);
    else
        launchDependent(postGatherKernel<R, false>, b, kThreads, 0, s, lam, lat, k, table, q, n, tmp);
    if (const int rc = checkLaunch("BC adjoint gather"))
        return rc;
    constexpr int V = VFB_BC_VELOCITY_INTERPOLATED, NS = VFB_BC_NOSLIP_INTERPOLATED;
    if (kind == V)
        (even ? launchPostScatter<R, V, true> : launchPostScatter<R, V, false>)(b, s, lam, lat, k, table, q, n, rec,
                                                                               tmp, gV);
    else
        (even ? launchPostScatter<R, NS, true> : launchPostScatter<R, NS, false>)(b, s, lam, lat, k, table, q, n, rec,
                                                                                 tmp, nullptr);
    return checkLaunch("BC adjoint scatter");
}

// first blocks of the lists of a multi-list launch; the total block count
template <class R>
int listBlocks(PostLists<R>& P, unsigned& blocks)
{
    if (P.count < 1 || P.count > kMaxPostLists)
        return setError(VFB_ERR_INVALID_ARGUMENT, "%d post-collision lists in one launch", P.count);
    blocks = 0;
    for (int l = 0; l < P.count; ++l) {
        const int kind = P.list[l].kind;
        if (kind != VFB_BC_VELOCITY_INTERPOLATED && kind != VFB_BC_NOSLIP_INTERPOLATED)
            return setError(VFB_ERR_INVALID_ARGUMENT, "BC kind %d has no adjoint", kind);
        P.firstBlock[l] = blocks;
        blocks += blocksFor(P.list[l].n);
    }
    return VFB_OK;
}

template <class R>
int postBCLists(R* dist, const BcLattice<R>& lat, PostLists<R> P, bool even, cudaStream_t s)
{
    unsigned b = 0;
    if (const int rc = listBlocks(P, b))
        return rc;
    if (b == 0)
        return VFB_OK;
    if (even)
        launchDependent(postBCListsKernel<R, true>, b, kThreads, 0, s, dist, lat, P);
    else
        launchDependent(postBCListsKernel<R, false>, b, kThreads, 0, s, dist, lat, P);
    return checkLaunch("adjoint forward BC lists");
}

template <class R>
int postBCAdjointLists(R* lam, const BcLattice<R>& lat, PostLists<R> P, bool even, cudaStream_t s)
{
    unsigned b = 0;
    if (const int rc = listBlocks(P, b))
        return rc;
    if (b == 0)
        return VFB_OK;
    if (even)
        launchDependent(postGatherListsKernel<R, true>, b, kThreads, 0, s, lam, lat, P);
    else
        launchDependent(postGatherListsKernel<R, false>, b, kThreads, 0, s, lam, lat, P);
    if (const int rc = checkLaunch("BC lists adjoint gather"))
        return rc;
    if (even)
        launchDependent(postScatterListsKernel<R, true>, b, kThreads, 0, s, lam, lat, P);
    else
        launchDependent(postScatterListsKernel<R, false>, b, kThreads, 0, s, lam, lat, P);
    return checkLaunch("BC lists adjoint scatter");
}

template <class R>
int pressureBC(R* dist, const BcLattice<R>& lat, const int32_t* k, const int32_t* kN, const R* rhoBC, uint32_t n,
               int direction, bool even, R* rec, cudaStream_t s)
{
    if (n == 0)
        return VFB_OK;
    int axis = 0, sgn = 0;
    if (const int rc = axisOf(direction, axis, sgn))
        return rc;
    const unsigned b = blocksFor(n);
    if (even)
        launchDependent(pressureKernel<R, true>, b, kThreads, 0, s, dist, lat, k, kN, rhoBC, n, axis, sgn, rec);
    else
        launchDependent(pressureKernel<R, false>, b, kThreads, 0, s, dist, lat, k, kN, rhoBC, n, axis, sgn, rec);
    return checkLaunch("adjoint forward pressure BC");
}

template <class R>
int pressureBCAdjoint(R* lam, const BcLattice<R>& lat, const int32_t* k, const int32_t* kN, const R* rhoBC,
                      uint32_t n, int direction, bool even, const R* rec, R* tmp, cudaStream_t s)
{
    if (n == 0)
        return VFB_OK;
    int axis = 0, sgn = 0;
    if (const int rc = axisOf(direction, axis, sgn))
        return rc;
    const unsigned b = blocksFor(n);
    if (even)
        launchDependent(pressureGatherKernel<R, true>, b, kThreads, 0, s, lam, lat, k, n, axis, sgn, tmp);
    else
        launchDependent(pressureGatherKernel<R, false>, b, kThreads, 0, s, lam, lat, k, n, axis, sgn, tmp);
    if (const int rc = checkLaunch("pressure adjoint gather"))
        return rc;
    if (even)
        launchDependent(pressureScatterKernel<R, true>, b, kThreads, 0, s, lam, lat, kN, rhoBC, n, axis, sgn, rec,
                        tmp);
    else
        launchDependent(pressureScatterKernel<R, false>, b, kThreads, 0, s, lam, lat, kN, rhoBC, n, axis, sgn, rec, tmp);
    return checkLaunch("pressure adjoint scatter");
}

template <class R>
int objective(const R* dist, unsigned long long N, const uint32_t* nX, const uint32_t* nY, const uint32_t* nZ,
              const uint32_t* nodes, const double* wx, const double* wy, const double* wz, uint32_t n, bool even,
              double* partials, R* lam, double seed, cudaStream_t s)
{
    if (n == 0)
        return VFB_OK;
    const unsigned b = blocksFor(n);
    if (even)
        objectiveKernel<R, true><<<b, kThreads, 0, s>>>(dist, N, nX, nY, nZ, nodes, wx, wy, wz, n, partials, lam,
                                                        seed);
    else
        objectiveKernel<R, false><<<b, kThreads, 0, s>>>(dist, N, nX, nY, nZ, nodes, wx, wy, wz, n, partials, lam,
                                                         seed);
    return checkLaunch("objective");
}

int reducePartials(const double* partials, unsigned blocks, int width, double* acc, double scale, cudaStream_t s)
{
    reduceKernel<<<width, kReduceThreads, 0, s>>>(partials, blocks, width, acc, scale);
    return checkLaunch("partial-sum reduction");
}

#define VFB_ADJOINT_INSTANTIATE(R)                                                                                    \
    template int collision<R>(R*, unsigned long long, const uint32_t*, const uint32_t*, const uint32_t*,             \
                              const uint32_t*, const uint32_t*, uint32_t, const K17Rates<R>&, R, R, R, bool, R*,     \
                              cudaStream_t);                                                                           \
    template int collisionAdjoint<R>(R*, unsigned long long, const uint32_t*, const uint32_t*, const uint32_t*,      \
                                     const uint32_t*, const uint32_t*, uint32_t, const K17Rates<R>&, R, R, R, bool,   \
                                     const R*, double*, cudaStream_t);                                                 \
    template int postBC<R>(int, R*, const BcLattice<R>&, const int32_t*, const uint32_t*, const R*, uint32_t,         \
                           const R*, const R*, const R*, bool, R*, cudaStream_t);                                      \
    template int postBCAdjoint<R>(int, R*, const BcLattice<R>&, const int32_t*, const uint32_t*, const R*, uint32_t,  \
                                  const R*, const R*, const R*, bool, const R*, R*, double*, cudaStream_t);            \
    template int postBCLists<R>(R*, const BcLattice<R>&, PostLists<R>, bool, cudaStream_t);                          \
    template int postBCAdjointLists<R>(R*, const BcLattice<R>&, PostLists<R>, bool, cudaStream_t);                   \
    template int pressureBC<R>(R*, const BcLattice<R>&, const int32_t*, const int32_t*, const R*, uint32_t, int,     \
                               bool, R*, cudaStream_t);                                                                \
    template int pressureBCAdjoint<R>(R*, const BcLattice<R>&, const int32_t*, const int32_t*, const R*, uint32_t,   \
                                      int, bool, const R*, R*, cudaStream_t);                                          \
    template int objective<R>(const R*, unsigned long long, const uint32_t*, const uint32_t*, const uint32_t*,       \
                              const uint32_t*, const double*, const double*, const double*, uint32_t, bool, double*,  \
                              R*, double, cudaStream_t);

VFB_ADJOINT_INSTANTIATE(float)
VFB_ADJOINT_INSTANTIATE(double)
#undef VFB_ADJOINT_INSTANTIATE

} // namespace adjoint
} // namespace vfb

using namespace vfb;

// Host check hook: the generated reverse sweep of one node on the host (the
// same code the collision adjoint kernel runs).  No counterpart in the
// reference.
extern "C" int vfb_debug_k17_adjoint_node(int precision, const double* f27, double* lam27, double omega,
                                          const double* limiters, const double* force, double* gforce3)
{
    clearError();
    if (!f27 || !lam27 || !limiters || !force || !gforce3)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    if (precision == VFB_FP64) {
        const K17Rates<double> r = makeK17Rates<double>(omega, limiters[0], limiters[1], limiters[2]);
        double a[27], l[27];
        for (int d = 0; d < 27; ++d) {
            a[d] = f27[d];
            l[d] = lam27[d];
        }
        k17Adjoint<double>(a, l, r, force[0], force[1], force[2], gforce3[0], gforce3[1], gforce3[2]);
        for (int d = 0; d < 27; ++d)
            lam27[d] = l[d];
        return VFB_OK;
    }
    if (precision == VFB_FP32) {
        const K17Rates<float> r = makeK17Rates<float>((float)omega, (float)limiters[0], (float)limiters[1],
                                                      (float)limiters[2]);
        float a[27], l[27], g[3];
        for (int d = 0; d < 27; ++d) {
            a[d] = (float)f27[d];
            l[d] = (float)lam27[d];
        }
        k17Adjoint<float>(a, l, r, (float)force[0], (float)force[1], (float)force[2], g[0], g[1], g[2]);
        for (int d = 0; d < 27; ++d)
            lam27[d] = l[d];
        for (int c = 0; c < 3; ++c)
            gforce3[c] = g[c];
        return VFB_OK;
    }
    return setError(VFB_ERR_INVALID_ARGUMENT, "precision must be VFB_FP64 or VFB_FP32");
}
