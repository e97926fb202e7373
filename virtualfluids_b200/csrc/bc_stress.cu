// bc_stress.cu -- the wall-model (stress) boundary conditions.
//
// StressCompressible_Device (StressCompressible.cu:50-762), StressBounceBack-
// Compressible_Device (StressBounceBackCompressible.cu:50-679) and StressBounce-
// BackPressureCompressible_Device (StressBounceBackPressureCompressible.cu),
// launched by StressCompressible / StressBounceBackCompressible /
// StressBounceBackPressureCompressible (Stress.cu:42-160) from
// BoundaryConditionKernelManager::runStressWallModelKernelPost
// (BoundaryConditionKernelManager.cpp:330-334), after the slip BC and before
// the geometry BC (UpdateGrid27.cpp:243-249).
//
// One thread per list entry, like the other BC kernels (bc.cu), with the
// entry's eight locations from the list's table when it has one.  Per entry:
//   1. the post-collision populations, drho and u (the plain BC sums);
//   2. for every wall direction (q in [0, 1], the reference's visiting order)
//      the incoming population of a wall at rest -- simple bounce-back,
//      bounce-back minus w drho, or the interpolated bounce-back with the
//      pressure term and the rate om / (1 + 3 om max(0, nu_t)) -- and the
//      momentum it exchanges with the wall;
//   3. the iMEM wall model (bc_math.cuh) turns that momentum and the filtered
//      velocities into a wall velocity (force factor 1, or 1 + q of the -z
//      direction for the interpolated kind) and advances both filters;
//   4. every incoming population gets the wall velocity's term 6 w c.U
//      (divided by 1 + q for the interpolated kind) and is written; the
//      monitor takes u* and the momentum including that term.
// StressCompressible_Device weighs the pressure term of its dPP0 direction
// with 2/27 instead of 1/54 (StressCompressible.cu:293); kept for parity.
#include <cuda_runtime.h>

#include "bc_math.cuh"
#include "capi_common.cuh"
#include "collision_math.cuh"
#include "d3q27.cuh"
#include "storage.cuh"
#include "pdl.cuh"

namespace vfb
{
namespace
{
template <class R>
struct StressArgs {
    const int32_t* __restrict__ k;
    const int32_t* __restrict__ kN;
    const R* __restrict__ q;
    const R* __restrict__ nx;
    const R* __restrict__ ny;
    const R* __restrict__ nz;
    R* __restrict__ el[3];
    R* __restrict__ wm[3];
    const int32_t* __restrict__ samplingOffset;
    const R* __restrict__ z0;
    R* __restrict__ uStar;
    R* __restrict__ F[3];
    const uint32_t* __restrict__ locations;
    const R* __restrict__ turb;
    const R* __restrict__ v[3]; // the level's macroscopic velocity, read at the sampling nodes
    uint32_t n;
};

template <class S, int KIND, bool EVEN>
__global__ void __launch_bounds__(128) bcStressKernel(S* __restrict__ dist, const BcLattice<typename Storage<S>::R> lat,
                                                       const StressArgs<typename Storage<S>::R> a)
{
    gridDependencyWait();
    using R = typename Storage<S>::R;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n)
        return;
    const unsigned long long N = lat.N;
    Locs L;
    if (a.locations) {
#pragma unroll
        for (int l = 0; l < 8; ++l)
            L.k[l] = __ldg(a.locations + (unsigned long long)l * a.n + i);
    } else {
        L = listIndices((uint32_t)__ldg(a.k + i), lat.nX, lat.nY, lat.nZ);
    }
    R g[27];
#pragma unroll
    for (int d = 0; d < 27; ++d)
        g[d] = Storage<S>::load(dist + (unsigned long long)slot<EVEN>(inv(d)) * N + L.k[loc(inv(d))], d);
    R qv[26];
#pragma unroll
    for (int j = 0; j < 26; ++j)
        qv[j] = __ldg(a.q + (unsigned long long)qOrder(j) * a.n + i);

    R drho, vx1, vx2, vx3;
    bcMacros(g, drho, vx1, vx2, vx3);
    const R cuSq = R(3) / R(2) * (vx1 * vx1 + vx2 * vx2 + vx3 * vx3) * (R(1) + drho);
    R om = lat.omega;
    if (KIND == VFB_BC_STRESS_INTERPOLATED && a.turb) {
        const R nu = __ldg(a.turb + __ldg(a.k + i));
        om = lat.omega / (R(1) + R(3) * lat.omega * fmax(R(0), nu));
    }

    // 2. incoming populations of a wall at rest and the exchanged momentum
    R fin[26];
    R mom[3] = { R(0), R(0), R(0) };
#pragma unroll
    for (int j = 0; j < 26; ++j) {
        const int d = qOrder(j);
        fin[j] = R(0);
        if (!(qv[j] >= R(0) && qv[j] <= R(1)))
            continue;
        const R w = weight<R>(d);
        if (KIND == VFB_BC_STRESS_BOUNCE_BACK) {
            fin[j] = g[d];
        } else if (KIND == VFB_BC_STRESS_BOUNCE_BACK_PRESSURE) {
            fin[j] = g[d] - w * drho;
        } else {
            const R feq = feqBC(drho, cdot<R>(d, vx1, vx2, vx3), cuSq, w);
            const R wp = d == dPP0 ? R(2) / R(27) : w;
            fin[j] = interpNoSlipPressure(qv[j], g[d], g[inv(d)], feq, om, drho, wp);
        }
        const R t = g[d] + fin[j];
        if (cx(d) > 0) mom[0] = mom[0] + t; else if (cx(d) < 0) mom[0] = mom[0] - t;
        if (cy(d) > 0) mom[1] = mom[1] + t; else if (cy(d) < 0) mom[1] = mom[1] - t;
        if (cz(d) > 0) mom[2] = mom[2] + t; else if (cz(d) < 0) mom[2] = mom[2] - t;
    }

    // 3. the wall model
    const R eps = R(0.001f);
    const uint32_t kN = (uint32_t)__ldg(a.kN + i);
    R el[3], wm[3];
    const R vw[3] = { vx1, vx2, vx3 };
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        el[c] = imemFilter(eps, __ldg(a.v[c] + kN), a.el[c][i]);
        wm[c] = imemFilter(eps, vw[c], a.wm[c][i]);
        a.el[c][i] = el[c];
        a.wm[c][i] = wm[c];
    }
    const R nrm[3] = { __ldg(a.nx + i), __ldg(a.ny + i), __ldg(a.nz + i) };
    const R qB = qv[5]; // q of d00M: qOrder(5)
    const R forceFactor = KIND == VFB_BC_STRESS_INTERPOLATED ? (R)(1.0 + (double)qB) : R(1);
    const R z = (R)__ldg(a.samplingOffset + i) + qB;
    R uStar, V[3];
    imemWallVelocity(nrm, el, wm, vw, R(1) + drho, z, __ldg(a.z0 + i), forceFactor, mom, uStar, V);

    // 4. the wall velocity's term, the writes and the monitor's momentum
#pragma unroll
    for (int j = 0; j < 26; ++j) {
        const int d = qOrder(j);
        if (!(qv[j] >= R(0) && qv[j] <= R(1)))
            continue;
        const int e = inv(d);
        R term = R(6) * weight<R>(d) * cdot<R>(d, V[0], V[1], V[2]);
        if (KIND == VFB_BC_STRESS_INTERPOLATED)
            term = term / (R(1) + qv[j]);
        Storage<S>::store(dist + (unsigned long long)slot<!EVEN>(e) * N + L.k[loc(e)], fin[j] - term, d);
        if (cx(d) > 0) mom[0] = mom[0] - term; else if (cx(d) < 0) mom[0] = mom[0] + term;
        if (cy(d) > 0) mom[1] = mom[1] - term; else if (cy(d) < 0) mom[1] = mom[1] + term;
        if (cz(d) > 0) mom[2] = mom[2] - term; else if (cz(d) < 0) mom[2] = mom[2] + term;
    }
    if (a.uStar) {
        a.uStar[i] = uStar;
        a.F[0][i] = mom[0];
        a.F[1][i] = mom[1];
        a.F[2][i] = mom[2];
    }
}

template <class S, int KIND>
void launchKind(bool even, unsigned blocks, cudaStream_t s, S* dist, const BcLattice<typename Storage<S>::R>& lat,
                const StressArgs<typename Storage<S>::R>& a)
{
    if (even)
        launchDependent(bcStressKernel<S, KIND, true>, blocks, 128, 0, s, dist, lat, a);
    else
        launchDependent(bcStressKernel<S, KIND, false>, blocks, 128, 0, s, dist, lat, a);
}

template <class S>
int launchStress(int kind, const vfb_bc_lattice* t, const vfb_stress_list* l, const void* turb, const void* vx,
                 const void* vy, const void* vz, cudaStream_t s)
{
    using R = typename Storage<S>::R;
    BcLattice<R> lat { t->numberOfLBnodes, t->neighborX, t->neighborY, t->neighborZ, (R)t->omega };
    StressArgs<R> a;
    a.k = l->k;
    a.kN = l->kN;
    a.q = static_cast<const R*>(l->q);
    a.nx = static_cast<const R*>(l->normalX);
    a.ny = static_cast<const R*>(l->normalY);
    a.nz = static_cast<const R*>(l->normalZ);
    a.el[0] = static_cast<R*>(l->Vx);
    a.el[1] = static_cast<R*>(l->Vy);
    a.el[2] = static_cast<R*>(l->Vz);
    a.wm[0] = static_cast<R*>(l->Vx1);
    a.wm[1] = static_cast<R*>(l->Vy1);
    a.wm[2] = static_cast<R*>(l->Vz1);
    a.samplingOffset = l->samplingOffset;
    a.z0 = static_cast<const R*>(l->z0);
    a.uStar = static_cast<R*>(l->uStar);
    a.F[0] = static_cast<R*>(l->Fx);
    a.F[1] = static_cast<R*>(l->Fy);
    a.F[2] = static_cast<R*>(l->Fz);
    a.locations = l->locations;
    a.turb = static_cast<const R*>(turb);
    a.v[0] = static_cast<const R*>(vx);
    a.v[1] = static_cast<const R*>(vy);
    a.v[2] = static_cast<const R*>(vz);
    a.n = l->numberOfBCnodes;
    S* dist = static_cast<S*>(t->distributions);
    const unsigned blocks = (a.n + 127) / 128;
    const bool even = t->isEvenTimestep != 0;
    switch (kind) {
    case VFB_BC_STRESS_INTERPOLATED: launchKind<S, VFB_BC_STRESS_INTERPOLATED>(even, blocks, s, dist, lat, a); break;
    case VFB_BC_STRESS_BOUNCE_BACK: launchKind<S, VFB_BC_STRESS_BOUNCE_BACK>(even, blocks, s, dist, lat, a); break;
    default: launchKind<S, VFB_BC_STRESS_BOUNCE_BACK_PRESSURE>(even, blocks, s, dist, lat, a); break;
    }
    return checkLaunch("stress boundary condition");
}
} // namespace
} // namespace vfb

using namespace vfb;

extern "C" int vfb_bc_stress(int kind, int storage, const vfb_bc_lattice* lattice, const vfb_stress_list* list,
                             const void* turbViscosity, const void* vx, const void* vy, const void* vz, void* stream)
{
    clearError();
    if (kind < VFB_BC_STRESS_INTERPOLATED || kind > VFB_BC_STRESS_BOUNCE_BACK_PRESSURE)
        return setError(VFB_ERR_INVALID_ARGUMENT, "unknown stress BC kind %d", kind);
    if (vfb_storage_bytes(storage) == 0)
        return setError(VFB_ERR_INVALID_ARGUMENT, "unknown storage %d", storage);
    if (!list)
        return setError(VFB_ERR_INVALID_ARGUMENT, "list is NULL");
    if (list->numberOfBCnodes == 0)
        return VFB_OK;
    if (!lattice || !lattice->distributions || !lattice->neighborX || !lattice->neighborY || !lattice->neighborZ)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL lattice or lattice array");
    if (lattice->numberOfLBnodes < 2)
        return setError(VFB_ERR_OUT_OF_RANGE, "numberOfLBnodes %llu < 2", lattice->numberOfLBnodes);
    const vfb_stress_list* l = list;
    if (!l->k || !l->kN || !l->q || !l->normalX || !l->normalY || !l->normalZ || !l->Vx || !l->Vy || !l->Vz ||
        !l->Vx1 || !l->Vy1 || !l->Vz1 || !l->samplingOffset || !l->z0)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL array of the stress list");
    if (!vx || !vy || !vz)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL macroscopic velocity array");
    const int monitors = (l->uStar != nullptr) + (l->Fx != nullptr) + (l->Fy != nullptr) + (l->Fz != nullptr);
    if (monitors != 0 && monitors != 4)
        return setError(VFB_ERR_INVALID_ARGUMENT, "the wall-model monitor needs uStar, Fx, Fy and Fz");
    if (kind == VFB_BC_STRESS_INTERPOLATED &&
        !(lattice->omega > 0.0 && lattice->omega < 2.0 && lattice->omega != 1.0))
        return setError(VFB_ERR_INVALID_ARGUMENT,
                        "omega %g outside (0, 2) or equal to 1 (the interpolation divides by 1 - omega)",
                        lattice->omega);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (storage) {
    case VFB_FP32: return launchStress<float>(kind, lattice, list, turbViscosity, vx, vy, vz, s);
    case VFB_FP64: return launchStress<double>(kind, lattice, list, turbViscosity, vx, vy, vz, s);
    case VFB_FP16: return launchStress<__half>(kind, lattice, list, turbViscosity, vx, vy, vz, s);
    case VFB_FX16: return launchStress<int16_t>(kind, lattice, list, turbViscosity, vx, vy, vz, s);
    case VFB_FX16W: return launchStress<fx16w_t>(kind, lattice, list, turbViscosity, vx, vy, vz, s);
    default: return launchStress<__nv_bfloat16>(kind, lattice, list, turbViscosity, vx, vy, vz, s);
    }
}
