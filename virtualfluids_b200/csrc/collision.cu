// collision.cu -- fused collide + esoteric-twist stream kernels (K17, BGK),
// equilibrium and non-equilibrium initialisation, macroscopic output and FP64
// reductions.
//
// One thread updates one fluid node: it follows the reference's index chain
// (ListIndices, src/gpu/core/Utilities/KernelUtilities.h:221-245) to the
// eight locations of the node, gathers the 27 pre-collision populations of the
// current parity (KernelUtilities.h:252-281), collides in registers and
// scatters the post-collision populations into the inverse slots
// (KernelUtilities.h:350-379).  Every location is read and written by exactly
// one thread, so the update is in place and race free.
#include <cuda_runtime.h>

#include <cstdio>

#include "capi_common.cuh"
#include "collision_math.cuh"
#include "d3q27.cuh"
#include "storage.cuh"
#include "pdl.cuh"

namespace vfb
{

template <class S>
struct CollisionKernelArgs {
    using R = typename Storage<S>::R;
    S* dist;
    S* base[27];          // dist + slot(d) * N for the parity of the launch
    unsigned long long N;
    const uint32_t* __restrict__ nX;
    const uint32_t* __restrict__ nY;
    const uint32_t* __restrict__ nZ;
    const uint32_t* __restrict__ fluid;
    uint32_t nFluid;
    // the list's location table (8 * nFluid, vfb_bc_locations layout) or null
    const uint32_t* __restrict__ table;
    K17Rates<R> rates;
    R fx, fy, fz;         // forces * 1/2 * forceFactor
    R gfx, gfy, gfz;      // raw global forces (body-force template)
    R forceFactor;
    R* rho;
    R* vx;
    R* vy;
    R* vz;
    R* bfx;
    R* bfy;
    R* bfz;
};

template <class S, bool EVEN>
__device__ __forceinline__ void gatherPre(typename Storage<S>::R* f, const S* __restrict__ dist, unsigned long long N,
                                          const Locs& L)
{
#pragma unroll
    for (int d = 0; d < 27; ++d)
        f[d] = Storage<S>::load(dist + (unsigned long long)slot<EVEN>(d) * N + L.k[loc(d)], d);
}

template <class S, bool EVEN>
__device__ __forceinline__ void scatterPost(const typename Storage<S>::R* f, S* __restrict__ dist, unsigned long long N,
                                            const Locs& L)
{
#pragma unroll
    for (int d = 0; d < 27; ++d)
        Storage<S>::store(dist + (unsigned long long)slot<EVEN>(d) * N + L.k[loc(d)], f[inv(d)], d);
}

template <class S, bool EVEN>
__device__ __forceinline__ void scatterPre(const typename Storage<S>::R* f, S* __restrict__ dist, unsigned long long N,
                                           const Locs& L)
{
#pragma unroll
    for (int d = 0; d < 27; ++d)
        Storage<S>::store(dist + (unsigned long long)slot<EVEN>(d) * N + L.k[loc(d)], f[d], d);
}

constexpr int kCollisionThreads = 128;

// the eight locations of list entry i (node k): from the list's location
// table in one round of independent loads, or through the neighbour chain
template <class S>
__device__ __forceinline__ Locs entryLocations(const CollisionKernelArgs<S>& a, uint32_t i, uint32_t k)
{
    if (a.table) {
        Locs L;
#pragma unroll
        for (int l = 0; l < 8; ++l)
            L.k[l] = __ldg(a.table + (unsigned long long)l * a.nFluid + i);
        return L;
    }
    return listIndices(k, a.nX, a.nY, a.nZ);
}

template <class S, bool EVEN, bool WRITE_MACRO, bool BODY_FORCE>
__global__ void __launch_bounds__(kCollisionThreads) k17Kernel(const CollisionKernelArgs<S> a)
{
    gridDependencyWait();
    using R = typename Storage<S>::R;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nFluid)
        return;
    const uint32_t k = __ldg(a.fluid + i);

    R fx = a.fx, fy = a.fy, fz = a.fz;
    if (BODY_FORCE) {
        fx = (a.gfx + a.bfx[k]) * R(0.5) * a.forceFactor;
        fy = (a.gfy + a.bfy[k]) * R(0.5) * a.forceFactor;
        fz = (a.gfz + a.bfz[k]) * R(0.5) * a.forceFactor;
        a.bfx[k] = R(0);
        a.bfy[k] = R(0);
        a.bfz[k] = R(0);
    }

    const Locs L = entryLocations(a, i, k);
    R f[27];
#pragma unroll
    for (int d = 0; d < 27; ++d)
        f[d] = Storage<S>::load(a.base[d] + L.k[loc(d)], d);
    R drho, ux, uy, uz;
    k17Collide<R>(f, a.rates, fx, fy, fz, drho, ux, uy, uz);
    if (WRITE_MACRO) {
        a.vx[k] = ux;
        a.vy[k] = uy;
        a.vz[k] = uz;
        a.rho[k] = drho;
    }
#pragma unroll
    for (int d = 0; d < 27; ++d)
        Storage<S>::store(a.base[d] + L.k[loc(d)], f[inv(d)], d);
}

template <class S, bool EVEN>
__global__ void __launch_bounds__(kCollisionThreads) bgkKernel(const CollisionKernelArgs<S> a)
{
    gridDependencyWait();
    using R = typename Storage<S>::R;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nFluid)
        return;
    const uint32_t k = __ldg(a.fluid + i);
    const Locs L = entryLocations(a, i, k);
    R f[27];
#pragma unroll
    for (int d = 0; d < 27; ++d)
        f[d] = Storage<S>::load(a.base[d] + L.k[loc(d)], d);
    bgkCollide<R>(f, a.rates.omega);
#pragma unroll
    for (int d = 0; d < 27; ++d)
        Storage<S>::store(a.base[d] + L.k[loc(d)], f[inv(d)], d);
}

// InitNavierStokesCompressible_Device.cu:173-200
template <class S, bool EVEN>
__global__ void initEqKernel(S* dist, unsigned long long N, const uint32_t* __restrict__ geo,
                             const uint32_t* __restrict__ nX, const uint32_t* __restrict__ nY,
                             const uint32_t* __restrict__ nZ, const typename Storage<S>::R* rho,
                             const typename Storage<S>::R* ux, const typename Storage<S>::R* uy,
                             const typename Storage<S>::R* uz)
{
    using R = typename Storage<S>::R;
    const unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N)
        return;
    const uint32_t g = geo[k];
    if (g == 15u || g == 16u)
        return;
    const R drho = rho[k], vx1 = ux[k], vx2 = uy[k], vx3 = uz[k];
    const R cu_sq = R(1.5) * (vx1 * vx1 + vx2 * vx2 + vx3 * vx3);
    R f[27];
    f[d000] = weight<R>(d000) * (drho - cu_sq * (R(1) + drho));
#pragma unroll
    for (int d = 1; d < 27; ++d) {
        const R cu = cdot<R>(d, vx1, vx2, vx3);
        f[d] = weight<R>(d) * (drho + (R(1) + drho) * (R(3) * cu + R(4.5) * cu * cu - cu_sq));
    }
    const Locs L = listIndices((uint32_t)k, nX, nY, nZ);
    scatterPre<S, EVEN>(f, dist, N, L);
}

// Non-equilibrium initialisation, InitNavierStokesCompressible_Device.cu:216-500.
// Opposite directions share one non-equilibrium coefficient (:460-486).
// Slots: 0 rest, 1-3 the x, y, z axes, 4 / 5 xy same / opposite signs, 6 / 7
// xz, 8 / 9 yz, 10 PPP/MMM, 11 PPM/MMP, 12 PMP/MPM, 13 PMM/MPP.
__host__ __device__ constexpr int noneqSlot(int d)
{
    constexpr int t[27] = { 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 8, 8, 9, 9, 10, 13, 12, 11, 11, 12, 13, 10 };
    return t[d];
}

// The fourteen first-order (strain-rate) non-equilibrium coefficients from the
// central-difference velocity gradient g[a][b] = d u_a / d x_b (:378-425).
// The reference writes them with double literals, so in its single-precision
// build too every product with a literal is a double product, sums of two
// gradients in parentheses stay in the working precision, and each
// coefficient is rounded to the working precision once; the code below keeps
// that, so FP32 follows that build.  The reference's factors eps_new and op
// are 1 and multiply exactly; they are left out.
template <class R>
__host__ __device__ inline void noneqCoefficients(const R g[3][3], R omega, R c[14])
{
    const R ax = g[0][0], ay = g[0][1], az = g[0][2];
    const R bx = g[1][0], by = g[1][1], bz = g[1][2];
    const R cx = g[2][0], cy = g[2][1], cz = g[2][2];
    const double o = (double)omega;
    const double five = 5.0 * o;
    c[1] = R((5.0 * ax * o + 5.0 * by * o + 5.0 * cz * o - 8.0 * ax + 4.0 * by + 4.0 * cz) / (54.0 * o));
    c[2] = R(c[1] + (2.0 * (ax - by)) / (9.0 * o));
    c[3] = R(c[1] + (2.0 * (ax - cz)) / (9.0 * o));
    c[4] = R(-(5.0 * cz * o + 3.0 * (ay + bx) - 2.0 * cz + ax * (five + 1.0) + by * (five + 1.0)) / (54.0 * o));
    c[5] = R(c[4] + (ay + bx) / (9.0 * o));
    c[6] = R(-(5.0 * cz * o + by * (five - 2.0) + 3.0 * (az + cx) + cz + ax * (five + 1.0)) / (54.0 * o));
    c[7] = R(c[6] + (az + cx) / (9.0 * o));
    c[8] = R(-(5.0 * ax * o + 5.0 * by * o + 5.0 * cz * o - 2.0 * ax + by + 3.0 * bz + 3.0 * cy + cz) / (54.0 * o));
    c[9] = R(c[8] + (bz + cy) / (9.0 * o));
    c[0] = R((5.0 * (ax + by + cz)) / 9.0);
    c[10] = R(-(ay + az + bx + bz + cx + cy) / (72.0 * o));
    c[11] = R(-c[10] - (ay + bx) / (36.0 * o));
    c[12] = R(-c[10] - (az + cx) / (36.0 * o));
    c[13] = R(-c[10] - (bz + cy) / (36.0 * o));
}

// equilibrium of (drho, u) plus (1 + drho) times each direction's
// non-equilibrium coefficient (:428-486), canonical direction order
template <class R>
__host__ __device__ inline void noneqNode(R drho, R vx1, R vx2, R vx3, const R g[3][3], R omega, R* f)
{
    R c[14];
    noneqCoefficients<R>(g, omega, c);
    const R cu_sq = R(1.5) * (vx1 * vx1 + vx2 * vx2 + vx3 * vx3);
    const R rho1 = R(1) + drho;
    f[d000] = weight<R>(d000) * (drho - cu_sq * rho1) + rho1 * c[0];
#pragma unroll
    for (int d = 1; d < 27; ++d) {
        const R cu = cdot<R>(d, vx1, vx2, vx3);
        const R eq = weight<R>(d) * (drho + rho1 * (R(3) * cu + R(4.5) * cu * cu - cu_sq));
        f[d] = eq + rho1 * c[noneqSlot(d)];
    }
}

// The reference sets the rest population of a solid or void node to 96
// (:490-499).  The scaled 16-bit formats cannot hold 96 (their ranges end near
// 16 and at 0.07), so they store their largest code instead.
template <class S>
__device__ __forceinline__ void storeSolidMarker(S* p)
{
    if constexpr (Storage<S>::scaled)
        Storage<S>::storeRaw(p, Storage<S>::marker);
    else
        Storage<S>::store(p, typename Storage<S>::R(96), d000);
}

template <class S, bool EVEN>
__global__ void initNoneqKernel(S* dist, unsigned long long N, const uint32_t* __restrict__ geo,
                                const uint32_t* __restrict__ nX, const uint32_t* __restrict__ nY,
                                const uint32_t* __restrict__ nZ, const uint32_t* __restrict__ nNeg,
                                const typename Storage<S>::R* rho, const typename Storage<S>::R* ux,
                                const typename Storage<S>::R* uy, const typename Storage<S>::R* uz,
                                typename Storage<S>::R omega)
{
    using R = typename Storage<S>::R;
    const unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N)
        return;
    const uint32_t type = geo[k];
    if (type == 15u || type == 16u) {
        storeSolidMarker<S>(dist + k);
        return;
    }
    // axis neighbours; the negative ones through the inverse (-x-y-z)
    // neighbour and two positive steps (:347-353)
    const uint32_t w = __ldg(nNeg + k);
    const uint32_t wx = __ldg(nX + w);
    const uint32_t plus[3] = { __ldg(nX + k), __ldg(nY + k), __ldg(nZ + k) };
    const uint32_t minus[3] = { __ldg(nZ + __ldg(nY + w)), __ldg(nZ + wx), __ldg(nY + wx) };
    const R* u[3] = { ux, uy, uz };
    R g[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
            g[a][b] = (u[a][plus[b]] - u[a][minus[b]]) / R(2);
    R f[27];
    noneqNode<R>(rho[k], ux[k], uy[k], uz[k], g, omega, f);
    const Locs L = listIndices((uint32_t)k, nX, nY, nZ);
    scatterPre<S, EVEN>(f, dist, N, L);
}

template <class S, bool EVEN>
__global__ void macroscopicKernel(const S* dist, unsigned long long N, const uint32_t* __restrict__ geo,
                                  const uint32_t* __restrict__ nX, const uint32_t* __restrict__ nY,
                                  const uint32_t* __restrict__ nZ, typename Storage<S>::R* rho,
                                  typename Storage<S>::R* vx, typename Storage<S>::R* vy, typename Storage<S>::R* vz)
{
    using R = typename Storage<S>::R;
    const unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N)
        return;
    const uint32_t g = geo[k];
    if (g == 15u || g == 16u) {
        rho[k] = R(0);
        vx[k] = R(0);
        vy[k] = R(0);
        vz[k] = R(0);
        return;
    }
    const Locs L = listIndices((uint32_t)k, nX, nY, nZ);
    R f[27];
    gatherPre<S, EVEN>(f, dist, N, L);
    const R drho = pyramidDensity(f);
    const R oneOverRho = R(1) / (drho + R(1));
    rho[k] = drho;
    vx[k] = pyramidJx(f) * oneOverRho;
    vy[k] = pyramidJy(f) * oneOverRho;
    vz[k] = pyramidJz(f) * oneOverRho;
}

// FP64 block partial sums of mass, kinetic energy and non-finite count
constexpr int kReduceThreads = 256;

template <class S, bool EVEN>
__global__ void __launch_bounds__(kReduceThreads) massEnergyKernel(const S* dist, unsigned long long N,
                                                                   const uint32_t* __restrict__ nX,
                                                                   const uint32_t* __restrict__ nY,
                                                                   const uint32_t* __restrict__ nZ,
                                                                   const uint32_t* __restrict__ idx, uint32_t n,
                                                                   double* __restrict__ partial)
{
    using R = typename Storage<S>::R;
    double m = 0.0, e = 0.0, bad = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k = __ldg(idx + i);
        const Locs L = listIndices(k, nX, nY, nZ);
        R f[27];
        gatherPre<S, EVEN>(f, dist, N, L);
        const R drho = pyramidDensity(f);
        const R oneOverRho = R(1) / (drho + R(1));
        const double ux = (double)(pyramidJx(f) * oneOverRho);
        const double uy = (double)(pyramidJy(f) * oneOverRho);
        const double uz = (double)(pyramidJz(f) * oneOverRho);
        const double ke = 0.5 * (ux * ux + uy * uy + uz * uz) * ((double)drho + 1.0);
        if (isfinite(ke) && isfinite((double)drho)) {
            m += (double)drho;
            e += ke;
        } else {
            bad += 1.0;
        }
    }
    // warp then block reduction
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        m += __shfl_down_sync(0xffffffffu, m, o);
        e += __shfl_down_sync(0xffffffffu, e, o);
        bad += __shfl_down_sync(0xffffffffu, bad, o);
    }
    __shared__ double sm[3][kReduceThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        sm[0][warp] = m;
        sm[1][warp] = e;
        sm[2][warp] = bad;
    }
    __syncthreads();
    if (warp == 0) {
        m = lane < kReduceThreads / 32 ? sm[0][lane] : 0.0;
        e = lane < kReduceThreads / 32 ? sm[1][lane] : 0.0;
        bad = lane < kReduceThreads / 32 ? sm[2][lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            m += __shfl_down_sync(0xffffffffu, m, o);
            e += __shfl_down_sync(0xffffffffu, e, o);
            bad += __shfl_down_sync(0xffffffffu, bad, o);
        }
        if (lane == 0) {
            partial[3 * blockIdx.x + 0] = m;
            partial[3 * blockIdx.x + 1] = e;
            partial[3 * blockIdx.x + 2] = bad;
        }
    }
}

// ------------------------------------------------------------- launchers --
template <class S>
static int launchCollision(bool bgk, const vfb_collision_args* a, cudaStream_t stream, const uint32_t* table = nullptr)
{
    using R = typename Storage<S>::R;
    CollisionKernelArgs<S> k;
    k.table = table;
    k.dist = static_cast<S*>(a->distributions);
    k.N = a->numberOfLBnodes;
    k.nX = a->neighborX;
    k.nY = a->neighborY;
    k.nZ = a->neighborZ;
    k.fluid = a->fluidNodeIndices;
    k.nFluid = a->numberOfFluidNodes;
    k.rates = makeK17Rates<R>((R)a->omega, (R)a->quadricLimiters[0], (R)a->quadricLimiters[1],
                              (R)a->quadricLimiters[2]);
    k.forceFactor = (R)a->forceFactor;
    k.gfx = (R)a->forces[0];
    k.gfy = (R)a->forces[1];
    k.gfz = (R)a->forces[2];
    k.fx = k.gfx * R(0.5) * k.forceFactor;
    k.fy = k.gfy * R(0.5) * k.forceFactor;
    k.fz = k.gfz * R(0.5) * k.forceFactor;
    k.rho = static_cast<R*>(a->rho);
    k.vx = static_cast<R*>(a->vx);
    k.vy = static_cast<R*>(a->vy);
    k.vz = static_cast<R*>(a->vz);
    k.bfx = static_cast<R*>(a->bodyForceX);
    k.bfy = static_cast<R*>(a->bodyForceY);
    k.bfz = static_cast<R*>(a->bodyForceZ);
    if (a->numberOfFluidNodes == 0)
        return VFB_OK;
    const unsigned blocks = (a->numberOfFluidNodes + kCollisionThreads - 1) / kCollisionThreads;
    const bool even = a->isEvenTimestep != 0;
    for (int d = 0; d < 27; ++d)
        k.base[d] = k.dist + (unsigned long long)(even ? d : inv(d)) * k.N;
    if (bgk) {
        if (even)
            launchDependent(bgkKernel<S, true>, blocks, kCollisionThreads, 0, stream, k);
        else
            launchDependent(bgkKernel<S, false>, blocks, kCollisionThreads, 0, stream, k);
        return checkLaunch("bgk collision");
    }
    const int t = a->collisionTemplate;
#define VFB_K17(E, W, B) launchDependent(k17Kernel<S, E, W, B>, blocks, kCollisionThreads, 0, stream, k)
    switch (t) {
    case VFB_TEMPLATE_DEFAULT: even ? VFB_K17(true, false, false) : VFB_K17(false, false, false); break;
    case VFB_TEMPLATE_WRITE_MACRO_VARS: even ? VFB_K17(true, true, false) : VFB_K17(false, true, false); break;
    case VFB_TEMPLATE_APPLY_BODY_FORCE: even ? VFB_K17(true, false, true) : VFB_K17(false, false, true); break;
    case VFB_TEMPLATE_ALL_FEATURES: even ? VFB_K17(true, true, true) : VFB_K17(false, true, true); break;
    default: return setError(VFB_ERR_INVALID_ARGUMENT, "invalid collisionTemplate %d", t);
    }
#undef VFB_K17
    return checkLaunch("k17 collision");
}

static int checkCollisionArgs(int storage, const vfb_collision_args* a, bool bgk)
{
    if (!a)
        return setError(VFB_ERR_INVALID_ARGUMENT, "args is NULL");
    if (vfb_storage_bytes(storage) == 0)
        return setError(VFB_ERR_INVALID_ARGUMENT, "unknown storage %d", storage);
    if (a->numberOfFluidNodes == 0)
        return VFB_OK;
    if (!a->distributions || !a->neighborX || !a->neighborY || !a->neighborZ || !a->fluidNodeIndices)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL distributions, neighbor or fluid-node array");
    if (a->numberOfLBnodes < 2 || a->numberOfLBnodes > 0xffffffffull)
        return setError(VFB_ERR_OUT_OF_RANGE, "numberOfLBnodes %llu outside [2, 2^32)", a->numberOfLBnodes);
    if (!(a->omega > 0.0 && a->omega < 2.0))
        return setError(VFB_ERR_INVALID_ARGUMENT, "omega %g outside (0, 2)", a->omega);
    if (!bgk) {
        const int t = a->collisionTemplate;
        if ((t == VFB_TEMPLATE_WRITE_MACRO_VARS || t == VFB_TEMPLATE_ALL_FEATURES) &&
            (!a->rho || !a->vx || !a->vy || !a->vz))
            return setError(VFB_ERR_INVALID_ARGUMENT, "template %d needs rho/vx/vy/vz", t);
        if ((t == VFB_TEMPLATE_APPLY_BODY_FORCE || t == VFB_TEMPLATE_ALL_FEATURES) &&
            (!a->bodyForceX || !a->bodyForceY || !a->bodyForceZ))
            return setError(VFB_ERR_INVALID_ARGUMENT, "template %d needs bodyForceX/Y/Z", t);
    }
    return VFB_OK;
}

template <class S>
static int launchInit(void* dist, unsigned long long N, const uint32_t* geo, const uint32_t* nX, const uint32_t* nY,
                      const uint32_t* nZ, const void* rho, const void* vx, const void* vy, const void* vz, int even,
                      cudaStream_t stream)
{
    using R = typename Storage<S>::R;
    const unsigned blocks = (unsigned)((N + 127) / 128);
    if (even)
        initEqKernel<S, true><<<blocks, 128, 0, stream>>>(static_cast<S*>(dist), N, geo, nX, nY, nZ,
                                                          static_cast<const R*>(rho), static_cast<const R*>(vx),
                                                          static_cast<const R*>(vy), static_cast<const R*>(vz));
    else
        initEqKernel<S, false><<<blocks, 128, 0, stream>>>(static_cast<S*>(dist), N, geo, nX, nY, nZ,
                                                           static_cast<const R*>(rho), static_cast<const R*>(vx),
                                                           static_cast<const R*>(vy), static_cast<const R*>(vz));
    return checkLaunch("init equilibrium");
}

template <class S>
static int launchInitNoneq(void* dist, unsigned long long N, const uint32_t* geo, const uint32_t* nX,
                           const uint32_t* nY, const uint32_t* nZ, const uint32_t* nNeg, const void* rho,
                           const void* vx, const void* vy, const void* vz, double omega, int even,
                           cudaStream_t stream)
{
    using R = typename Storage<S>::R;
    const unsigned blocks = (unsigned)((N + 127) / 128);
    const R* f[4] = { static_cast<const R*>(rho), static_cast<const R*>(vx), static_cast<const R*>(vy),
                      static_cast<const R*>(vz) };
    if (even)
        initNoneqKernel<S, true><<<blocks, 128, 0, stream>>>(static_cast<S*>(dist), N, geo, nX, nY, nZ, nNeg, f[0],
                                                             f[1], f[2], f[3], (R)omega);
    else
        initNoneqKernel<S, false><<<blocks, 128, 0, stream>>>(static_cast<S*>(dist), N, geo, nX, nY, nZ, nNeg, f[0],
                                                              f[1], f[2], f[3], (R)omega);
    return checkLaunch("init non-equilibrium");
}

template <class S>
static int launchMacro(const void* dist, unsigned long long N, const uint32_t* geo, const uint32_t* nX,
                       const uint32_t* nY, const uint32_t* nZ, int even, void* rho, void* vx, void* vy, void* vz,
                       cudaStream_t stream)
{
    using R = typename Storage<S>::R;
    const unsigned blocks = (unsigned)((N + 127) / 128);
    if (even)
        macroscopicKernel<S, true><<<blocks, 128, 0, stream>>>(static_cast<const S*>(dist), N, geo, nX, nY, nZ,
                                                               static_cast<R*>(rho), static_cast<R*>(vx),
                                                               static_cast<R*>(vy), static_cast<R*>(vz));
    else
        macroscopicKernel<S, false><<<blocks, 128, 0, stream>>>(static_cast<const S*>(dist), N, geo, nX, nY, nZ,
                                                                static_cast<R*>(rho), static_cast<R*>(vx),
                                                                static_cast<R*>(vy), static_cast<R*>(vz));
    return checkLaunch("macroscopic");
}

template <class S>
static int launchMassEnergy(const void* dist, unsigned long long N, const uint32_t* nX, const uint32_t* nY,
                            const uint32_t* nZ, const uint32_t* idx, uint32_t n, int even, double* partial,
                            unsigned blocks, cudaStream_t stream)
{
    if (even)
        massEnergyKernel<S, true><<<blocks, kReduceThreads, 0, stream>>>(static_cast<const S*>(dist), N, nX, nY, nZ,
                                                                         idx, n, partial);
    else
        massEnergyKernel<S, false><<<blocks, kReduceThreads, 0, stream>>>(static_cast<const S*>(dist), N, nX, nY,
                                                                          nZ, idx, n, partial);
    return checkLaunch("mass and energy");
}

} // namespace vfb

using namespace vfb;

extern "C" int vfb_k17_collision(int storage, const vfb_collision_args* args, void* stream)
{
    clearError();
    int rc = checkCollisionArgs(storage, args, false);
    if (rc != VFB_OK || args->numberOfFluidNodes == 0)
        return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (storage) {
    case VFB_FP32: return launchCollision<float>(false, args, s);
    case VFB_FP64: return launchCollision<double>(false, args, s);
    case VFB_FP16: return launchCollision<__half>(false, args, s);
    case VFB_FX16: return launchCollision<int16_t>(false, args, s);
    case VFB_FX16W: return launchCollision<fx16w_t>(false, args, s);
    case VFB_BF16: return launchCollision<__nv_bfloat16>(false, args, s);
    default: return setError(VFB_ERR_INVALID_ARGUMENT, "unknown storage %d", storage);
    }
}

namespace vfb
{
int laneCollision(int storage, bool bgk, const vfb_collision_args* args, const uint32_t* table, void* stream)
{
    int rc = checkCollisionArgs(storage, args, bgk);
    if (rc != VFB_OK || args->numberOfFluidNodes == 0)
        return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (storage) {
    case VFB_FP32: return launchCollision<float>(bgk, args, s, table);
    case VFB_FP64: return launchCollision<double>(bgk, args, s, table);
    case VFB_FP16: return launchCollision<__half>(bgk, args, s, table);
    case VFB_FX16: return launchCollision<int16_t>(bgk, args, s, table);
    case VFB_FX16W: return launchCollision<fx16w_t>(bgk, args, s, table);
    case VFB_BF16: return launchCollision<__nv_bfloat16>(bgk, args, s, table);
    default: return setError(VFB_ERR_INVALID_ARGUMENT, "unknown storage %d", storage);
    }
}
} // namespace vfb

extern "C" int vfb_bgk_collision(int storage, const vfb_collision_args* args, void* stream)
{
    clearError();
    int rc = checkCollisionArgs(storage, args, true);
    if (rc != VFB_OK || args->numberOfFluidNodes == 0)
        return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (storage) {
    case VFB_FP32: return launchCollision<float>(true, args, s);
    case VFB_FP64: return launchCollision<double>(true, args, s);
    case VFB_FP16: return launchCollision<__half>(true, args, s);
    case VFB_FX16: return launchCollision<int16_t>(true, args, s);
    case VFB_FX16W: return launchCollision<fx16w_t>(true, args, s);
    case VFB_BF16: return launchCollision<__nv_bfloat16>(true, args, s);
    default: return setError(VFB_ERR_INVALID_ARGUMENT, "unknown storage %d", storage);
    }
}

extern "C" int vfb_init_equilibrium(int storage, void* distributions, unsigned long long N, const uint32_t* geo,
                                    const uint32_t* nX, const uint32_t* nY, const uint32_t* nZ, const void* rho,
                                    const void* vx, const void* vy, const void* vz, int isEven, void* stream)
{
    clearError();
    if (!distributions || !geo || !nX || !nY || !nZ || !rho || !vx || !vy || !vz)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    if (N < 2 || N > 0xffffffffull)
        return setError(VFB_ERR_OUT_OF_RANGE, "numberOfLBnodes %llu outside [2, 2^32)", N);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (storage) {
    case VFB_FP32: return launchInit<float>(distributions, N, geo, nX, nY, nZ, rho, vx, vy, vz, isEven, s);
    case VFB_FP64: return launchInit<double>(distributions, N, geo, nX, nY, nZ, rho, vx, vy, vz, isEven, s);
    case VFB_FP16: return launchInit<__half>(distributions, N, geo, nX, nY, nZ, rho, vx, vy, vz, isEven, s);
    case VFB_FX16: return launchInit<int16_t>(distributions, N, geo, nX, nY, nZ, rho, vx, vy, vz, isEven, s);
    case VFB_FX16W: return launchInit<fx16w_t>(distributions, N, geo, nX, nY, nZ, rho, vx, vy, vz, isEven, s);
    case VFB_BF16: return launchInit<__nv_bfloat16>(distributions, N, geo, nX, nY, nZ, rho, vx, vy, vz, isEven, s);
    default: return setError(VFB_ERR_INVALID_ARGUMENT, "unknown storage %d", storage);
    }
}

extern "C" int vfb_init_nonequilibrium(int storage, void* distributions, unsigned long long N, const uint32_t* geo,
                                       const uint32_t* nX, const uint32_t* nY, const uint32_t* nZ,
                                       const uint32_t* neighborInverse, const void* rho, const void* vx, const void* vy,
                                       const void* vz, double omega, int isEven, void* stream)
{
    clearError();
    if (!distributions || !geo || !nX || !nY || !nZ || !neighborInverse || !rho || !vx || !vy || !vz)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    if (N < 2 || N > 0xffffffffull)
        return setError(VFB_ERR_OUT_OF_RANGE, "numberOfLBnodes %llu outside [2, 2^32)", N);
    if (!(omega > 0.0 && omega < 2.0))
        return setError(VFB_ERR_INVALID_ARGUMENT, "omega %g outside (0, 2)", omega);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint32_t* w = neighborInverse;
    switch (storage) {
    case VFB_FP32: return launchInitNoneq<float>(distributions, N, geo, nX, nY, nZ, w, rho, vx, vy, vz, omega, isEven, s);
    case VFB_FP64: return launchInitNoneq<double>(distributions, N, geo, nX, nY, nZ, w, rho, vx, vy, vz, omega, isEven, s);
    case VFB_FP16: return launchInitNoneq<__half>(distributions, N, geo, nX, nY, nZ, w, rho, vx, vy, vz, omega, isEven, s);
    case VFB_FX16: return launchInitNoneq<int16_t>(distributions, N, geo, nX, nY, nZ, w, rho, vx, vy, vz, omega, isEven, s);
    case VFB_FX16W: return launchInitNoneq<fx16w_t>(distributions, N, geo, nX, nY, nZ, w, rho, vx, vy, vz, omega, isEven, s);
    case VFB_BF16:
        return launchInitNoneq<__nv_bfloat16>(distributions, N, geo, nX, nY, nZ, w, rho, vx, vy, vz, omega, isEven, s);
    default: return setError(VFB_ERR_INVALID_ARGUMENT, "unknown storage %d", storage);
    }
}

extern "C" int vfb_macroscopic(int storage, const void* distributions, unsigned long long N, const uint32_t* geo,
                               const uint32_t* nX, const uint32_t* nY, const uint32_t* nZ, int isEven, void* rho,
                               void* vx, void* vy, void* vz, void* stream)
{
    clearError();
    if (!distributions || !geo || !nX || !nY || !nZ || !rho || !vx || !vy || !vz)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    if (N < 2 || N > 0xffffffffull)
        return setError(VFB_ERR_OUT_OF_RANGE, "numberOfLBnodes %llu outside [2, 2^32)", N);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (storage) {
    case VFB_FP32: return launchMacro<float>(distributions, N, geo, nX, nY, nZ, isEven, rho, vx, vy, vz, s);
    case VFB_FP64: return launchMacro<double>(distributions, N, geo, nX, nY, nZ, isEven, rho, vx, vy, vz, s);
    case VFB_FP16: return launchMacro<__half>(distributions, N, geo, nX, nY, nZ, isEven, rho, vx, vy, vz, s);
    case VFB_FX16: return launchMacro<int16_t>(distributions, N, geo, nX, nY, nZ, isEven, rho, vx, vy, vz, s);
    case VFB_FX16W: return launchMacro<fx16w_t>(distributions, N, geo, nX, nY, nZ, isEven, rho, vx, vy, vz, s);
    case VFB_BF16: return launchMacro<__nv_bfloat16>(distributions, N, geo, nX, nY, nZ, isEven, rho, vx, vy, vz, s);
    default: return setError(VFB_ERR_INVALID_ARGUMENT, "unknown storage %d", storage);
    }
}

// stored FX16 / FX16W codes at either end of the int16 range in slots 1..26 (slot 0,
// the rest population, also holds the solid-node marker); one 64-bit count
// per block, added with one atomic per block
__global__ void __launch_bounds__(kReduceThreads)
    saturationKernel(const int16_t* __restrict__ dist, unsigned long long begin, unsigned long long end,
                     unsigned long long* __restrict__ count)
{
    __shared__ unsigned long long part[kReduceThreads / 32];
    unsigned long long c = 0;
    for (unsigned long long i = begin + blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < end;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const int16_t q = __ldg(dist + i);
        c += (q == 32767 || q == -32768) ? 1u : 0u;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0)
        part[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < kReduceThreads / 32; ++w)
            t += part[w];
        if (t)
            atomicAdd(count, t);
    }
}

extern "C" int vfb_saturated_populations(int storage, const void* distributions, unsigned long long N,
                                         unsigned long long* count, void* stream)
{
    clearError();
    if (!count)
        return setError(VFB_ERR_INVALID_ARGUMENT, "count is NULL");
    *count = 0;
    if (vfb_storage_bytes(storage) == 0)
        return setError(VFB_ERR_INVALID_ARGUMENT, "unknown storage %d", storage);
    if ((storage != VFB_FX16 && storage != VFB_FX16W) || N == 0)
        return VFB_OK;
    if (!distributions)
        return setError(VFB_ERR_INVALID_ARGUMENT, "distributions is NULL");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int device = 0, sms = 148;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    unsigned long long* d = nullptr;
    if (cudaMallocAsync(&d, sizeof(unsigned long long), s) != cudaSuccess)
        return setError(VFB_ERR_CUDA, "cudaMallocAsync of the counter failed");
    int rc = VFB_OK;
    if (cudaMemsetAsync(d, 0, sizeof(unsigned long long), s) != cudaSuccess)
        rc = setError(VFB_ERR_CUDA, "counter clear failed");
    if (rc == VFB_OK) {
        saturationKernel<<<(unsigned)sms * 4u, kReduceThreads, 0, s>>>(static_cast<const int16_t*>(distributions), N,
                                                                       27ull * N, d);
        rc = checkLaunch("saturation count");
    }
    if (rc == VFB_OK && (cudaMemcpyAsync(count, d, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s) !=
                             cudaSuccess ||
                         cudaStreamSynchronize(s) != cudaSuccess))
        rc = setError(VFB_ERR_CUDA, "saturation count: %s", cudaGetErrorString(cudaGetLastError()));
    cudaFreeAsync(d, s);
    return rc;
}

extern "C" int vfb_mass_and_energy(int storage, const void* distributions, unsigned long long N, const uint32_t* nX,
                                   const uint32_t* nY, const uint32_t* nZ, const uint32_t* idx, uint32_t n,
                                   int isEven, double* out, void* stream)
{
    clearError();
    if (!out)
        return setError(VFB_ERR_INVALID_ARGUMENT, "out is NULL");
    out[0] = out[1] = out[2] = 0.0;
    if (n == 0)
        return VFB_OK;
    if (!distributions || !nX || !nY || !nZ || !idx)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    if (vfb_storage_bytes(storage) == 0)
        return setError(VFB_ERR_INVALID_ARGUMENT, "unknown storage %d", storage);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int device = 0, sms = 148;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    unsigned blocks = (unsigned)sms * 4u;
    const unsigned need = (n + kReduceThreads - 1) / kReduceThreads;
    if (need < blocks)
        blocks = need;
    double* partial = nullptr;
    if (cudaMallocAsync(&partial, sizeof(double) * 3 * blocks, s) != cudaSuccess)
        return setError(VFB_ERR_CUDA, "cudaMallocAsync of %u partial sums failed", blocks);
    int rc = VFB_OK;
    switch (storage) {
    case VFB_FP32: rc = launchMassEnergy<float>(distributions, N, nX, nY, nZ, idx, n, isEven, partial, blocks, s); break;
    case VFB_FP64: rc = launchMassEnergy<double>(distributions, N, nX, nY, nZ, idx, n, isEven, partial, blocks, s); break;
    case VFB_FP16: rc = launchMassEnergy<__half>(distributions, N, nX, nY, nZ, idx, n, isEven, partial, blocks, s); break;
    case VFB_FX16: rc = launchMassEnergy<int16_t>(distributions, N, nX, nY, nZ, idx, n, isEven, partial, blocks, s); break;
    case VFB_FX16W: rc = launchMassEnergy<fx16w_t>(distributions, N, nX, nY, nZ, idx, n, isEven, partial, blocks, s); break;
    default: rc = launchMassEnergy<__nv_bfloat16>(distributions, N, nX, nY, nZ, idx, n, isEven, partial, blocks, s); break;
    }
    if (rc == VFB_OK) {
        std::vector<double> host(3 * (size_t)blocks);
        if (cudaMemcpyAsync(host.data(), partial, sizeof(double) * 3 * blocks, cudaMemcpyDeviceToHost, s) !=
                cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            rc = setError(VFB_ERR_CUDA, "copy of partial sums failed: %s", cudaGetErrorString(cudaGetLastError()));
        } else {
            for (unsigned b = 0; b < blocks; ++b) {
                out[0] += host[3 * b + 0];
                out[1] += host[3 * b + 1];
                out[2] += host[3 * b + 2];
            }
        }
    }
    cudaFreeAsync(partial, s);
    return rc;
}

/*
 * One node of the K17 (op 0) or BGK (op 1) collision evaluated on the host
 * with the library's arithmetic (the same __host__ __device__ code the
 * kernels run; the host compiler does not contract multiply-adds beyond the
 * explicit fma calls).  precision: VFB_FP64 or VFB_FP32.  f27 in/out;
 * out4 = drho, vx, vy, vz (K17 only).  For tests without a GPU.
 */
extern "C" int vfb_debug_collide_node(int op, int precision, double* f27, double omega, const double* limiters,
                                      const double* force, double* out4)
{
    clearError();
    if (!f27 || !limiters || !force || !out4)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    if (precision == VFB_FP64) {
        double f[27];
        for (int d = 0; d < 27; ++d)
            f[d] = f27[d];
        const K17Rates<double> r = makeK17Rates<double>(omega, limiters[0], limiters[1], limiters[2]);
        if (op == 0)
            k17Collide<double>(f, r, force[0], force[1], force[2], out4[0], out4[1], out4[2], out4[3]);
        else
            bgkCollide<double>(f, omega);
        for (int d = 0; d < 27; ++d)
            f27[d] = f[d];
        return VFB_OK;
    }
    if (precision == VFB_FP32) {
        float f[27];
        for (int d = 0; d < 27; ++d)
            f[d] = (float)f27[d];
        const K17Rates<float> r = makeK17Rates<float>((float)omega, (float)limiters[0], (float)limiters[1],
                                                      (float)limiters[2]);
        float o[4] = { 0, 0, 0, 0 };
        if (op == 0)
            k17Collide<float>(f, r, (float)force[0], (float)force[1], (float)force[2], o[0], o[1], o[2], o[3]);
        else
            bgkCollide<float>(f, (float)omega);
        for (int d = 0; d < 27; ++d)
            f27[d] = f[d];
        for (int i = 0; i < 4; ++i)
            out4[i] = o[i];
        return VFB_OK;
    }
    return setError(VFB_ERR_INVALID_ARGUMENT, "precision must be VFB_FP64 or VFB_FP32");
}

namespace
{
template <class R>
void noneqNodeHost(const double* drhoVelocity4, const double* gradient9, double omega, double* f27)
{
    R g[3][3], f[27];
    for (int i = 0; i < 9; ++i)
        g[i / 3][i % 3] = (R)gradient9[i];
    noneqNode<R>((R)drhoVelocity4[0], (R)drhoVelocity4[1], (R)drhoVelocity4[2], (R)drhoVelocity4[3], g, (R)omega, f);
    for (int d = 0; d < 27; ++d)
        f27[d] = f[d];
}
} // namespace

/*
 * One node of the non-equilibrium initialisation evaluated on the host with
 * the code the kernel runs: drhoVelocity4 = drho, vx, vy, vz; gradient9[3a+b]
 * = d u_a / d x_b; f27 = the 27 populations in direction order.  precision:
 * VFB_FP64 or VFB_FP32 (inputs are rounded to it).  For tests without a GPU.
 */
extern "C" int vfb_debug_init_nonequilibrium_node(int precision, const double* drhoVelocity4, const double* gradient9,
                                                  double omega, double* f27)
{
    clearError();
    if (!drhoVelocity4 || !gradient9 || !f27)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    if (precision == VFB_FP64)
        noneqNodeHost<double>(drhoVelocity4, gradient9, omega, f27);
    else if (precision == VFB_FP32)
        noneqNodeHost<float>(drhoVelocity4, gradient9, omega, f27);
    else
        return setError(VFB_ERR_INVALID_ARGUMENT, "precision must be VFB_FP64 or VFB_FP32");
    return VFB_OK;
}
