// bc.cu -- boundary-condition kernels over compacted BC lists.
//
// One thread per BC node, as in the reference: the lists are small (a few
// planes of a level), so these kernels are bound by launch latency and the
// gather of the node's 27 populations, not by bandwidth.  The q array is
// direction-major, so the 26 q reads of a warp are coalesced.
//
// Post-collision kinds (run after the collision of the same parity, reading
// the post-collision values through the isEven view and writing the
// bounced-back values into the !isEven view, NoSlipInterpolatedCompressible.cu:71,165):
//   no-slip interpolated  NoSlipInterpolatedCompressible.cu:44-378
//   no-slip bounce-back   NoSlipBounceBack.cu
//   velocity interpolated VelocityInterpolatedCompressible.cu:44-418
//   velocity bounce-back  VelocityBounceBack.cu
//   slip                  SlipCompressible.cu:45-550
//   velocity with pressure VelocityWithPressureInterpolatedCompressible.cu
//                          (the velocity formula minus w drho, KernelUtilities.h:208-214)
// Pre-collision kinds (after the parity swap):
//   pressure non-equilibrium PressureNonEquilibriumCompressible.cu:45-311
//   non-reflecting outflow   OutflowNonReflecting.cu:50-276, with pressure
//                            correction OutflowNonReflectingPressureCorrection.cu:51-241
//
// Every node writes only its own locations, so no two nodes write one cell
// (for a fixed location bit the map node -> location index is one to one).
// Nodes of a list that are lattice neighbours of each other (around a solid
// body, not along a flat wall) can read a cell another node writes: a node's
// bounce-back value lands where a neighbouring BC node reads a post-collision
// population.  Like the reference's kernels, these read all of a node's values
// before writing, so a list resident in one wave sees the state before the
// launch everywhere; across waves the outcome depends on the schedule, as it
// does in the reference.
#include <cuda_runtime.h>

#include <cmath>

#include "bc_entry.cuh"
#include "bc_math.cuh"
#include "capi_common.cuh"
#include "collision_math.cuh"
#include "d3q27.cuh"
#include "storage.cuh"
#include "pdl.cuh"

namespace vfb
{

// the eight locations of entry i: from the list's location table when it has
// one (eight independent loads), else through the neighbour arrays
__device__ __forceinline__ Locs bcLocations(const uint32_t* __restrict__ table, uint32_t i, uint32_t n,
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

__global__ void bcLocationsKernel(const int32_t* __restrict__ bcK, uint32_t n, const uint32_t* __restrict__ nX,
                                  const uint32_t* __restrict__ nY, const uint32_t* __restrict__ nZ,
                                  uint32_t* __restrict__ out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const Locs L = listIndices((uint32_t)__ldg(bcK + i), nX, nY, nZ);
#pragma unroll
    for (int l = 0; l < 8; ++l)
        out[(unsigned long long)l * n + i] = L.k[l];
}

// six resident blocks of 128 threads: the gathers of a wall entry are DRAM
// bursts, so more of them in flight matter more than the few registers the
// 80-register bound spills
template <class S, int KIND, bool EVEN>
__global__ void __launch_bounds__(128, 6) bcPostKernel(S* __restrict__ dist, const BcLattice<typename Storage<S>::R> lat,
                                                     const int32_t* __restrict__ bcK,
                                                     const typename Storage<S>::R* __restrict__ q, uint32_t nBC,
                                                     const typename Storage<S>::R* __restrict__ Vx,
                                                     const typename Storage<S>::R* __restrict__ Vy,
                                                     const typename Storage<S>::R* __restrict__ Vz,
                                                     const uint32_t* __restrict__ locations)
{
    gridDependencyWait();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nBC)
        return;
    const Locs L = bcLocations(locations, i, nBC, bcK, lat.nX, lat.nY, lat.nZ);
    bcPostEntry<S, KIND, EVEN>(dist, lat.N, lat.omega, L, q, nBC, i, Vx, Vy, Vz);
}

// PressureNonEquilibriumCompressible.cu:75-309: the neighbour's
// pre-collision populations with their equilibrium part moved from the
// neighbour's density to the prescribed one, written into the BC node's
// directions whose component along the normal axis differs from the normal's
template <class S, bool EVEN>
__global__ void __launch_bounds__(128) bcPressureKernel(S* __restrict__ dist, const BcLattice<typename Storage<S>::R> lat,
                                                         const int32_t* __restrict__ bcK,
                                                         const int32_t* __restrict__ bcKN,
                                                         const typename Storage<S>::R* __restrict__ rhoBC, uint32_t nBC,
                                                         int axis, int sgn, const uint32_t* __restrict__ locations)
{
    gridDependencyWait();
    using R = typename Storage<S>::R;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nBC)
        return;
    const unsigned long long N = lat.N;
    // the BC node's and its neighbour's locations: from the list's table
    // (16 * nBC, the node's eight then the neighbour's) or through the chain
    Locs L, LN;
    if (locations) {
#pragma unroll
        for (int l = 0; l < 8; ++l) {
            L.k[l] = __ldg(locations + (unsigned long long)l * nBC + i);
            LN.k[l] = __ldg(locations + (unsigned long long)(8 + l) * nBC + i);
        }
    } else {
        L = listIndices((uint32_t)__ldg(bcK + i), lat.nX, lat.nY, lat.nZ);
        LN = listIndices((uint32_t)__ldg(bcKN + i), lat.nX, lat.nY, lat.nZ);
    }
    R f[27];
#pragma unroll
    for (int d = 0; d < 27; ++d)
        f[d] = Storage<S>::load(dist + (unsigned long long)slot<EVEN>(d) * N + LN.k[loc(d)], d);
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
        Storage<S>::store(dist + (unsigned long long)slot<EVEN>(d) * N + L.k[loc(d)], f[d], d);
    }
}

// OutflowNonReflecting.cu:50-276 (CORRECTION false) and
// OutflowNonReflectingPressureCorrection.cu:51-241 (true): for the nine
// directions whose component along the normal's axis is opposite to the
// normal, the BC node's population becomes cs f_neighbour + (1 - cs) f_node
// (minus w_d factor drho_node with the correction), read from the current
// view and written into the other one at the same location.  The corrected
// form takes the neighbour's shifted locations from the BC node (:89-96), so
// only its rest location is the neighbour's own; that is kept.  Reads (the
// nine directions) and writes (their inverse slots) never share a slot, so
// BC nodes of one list do not race.
template <class S, bool EVEN, bool CORRECTION>
__global__ void __launch_bounds__(128) bcOutflowKernel(S* __restrict__ dist, const BcLattice<typename Storage<S>::R> lat,
                                                        const int32_t* __restrict__ bcK,
                                                        const int32_t* __restrict__ bcKN, uint32_t nBC, int axis,
                                                        int sgn, typename Storage<S>::R cs,
                                                        typename Storage<S>::R factor)
{
    gridDependencyWait();
    using R = typename Storage<S>::R;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nBC)
        return;
    const unsigned long long N = lat.N;
    const Locs L = listIndices((uint32_t)__ldg(bcK + i), lat.nX, lat.nY, lat.nZ);
    Locs LN = L;
    if (CORRECTION)
        LN.k[0] = (uint32_t)__ldg(bcKN + i);
    else
        LN = listIndices((uint32_t)__ldg(bcKN + i), lat.nX, lat.nY, lat.nZ);
    R rhoCorrection = R(0);
    if (CORRECTION) {
        R f[27];
#pragma unroll
        for (int d = 0; d < 27; ++d)
            f[d] = Storage<S>::load(dist + (unsigned long long)slot<EVEN>(d) * N + L.k[loc(d)], d);
        rhoCorrection = factor * pyramidDensity(f);
    }
#pragma unroll
    for (int d = 1; d < 27; ++d) {
        const int c = axis == 0 ? cx(d) : axis == 1 ? cy(d) : cz(d);
        if (c != -sgn)
            continue;
        const R fNode = Storage<S>::load(dist + (unsigned long long)slot<EVEN>(d) * N + L.k[loc(d)], d);
        const R fNeighbour = Storage<S>::load(dist + (unsigned long long)slot<EVEN>(d) * N + LN.k[loc(d)], d);
        R v = fNeighbour * cs + (R(1) - cs) * fNode;
        if (CORRECTION)
            v = v - weight<R>(d) * rhoCorrection;
        Storage<S>::store(dist + (unsigned long long)slot<!EVEN>(d) * N + L.k[loc(d)], v, d);
    }
}

template <class S, int KIND>
static void launchPostKind(bool even, unsigned blocks, cudaStream_t stream, S* dist, const BcLattice<typename Storage<S>::R>& lat,
                           const vfb_bc_list* l)
{
    using R = typename Storage<S>::R;
    const R* q = static_cast<const R*>(l->q);
    const R* vx = static_cast<const R*>(l->Vx);
    const R* vy = static_cast<const R*>(l->Vy);
    const R* vz = static_cast<const R*>(l->Vz);
    if (even)
        launchDependent(bcPostKernel<S, KIND, true>, blocks, 128, 0, stream, dist, lat,
                        l->k, q, l->numberOfBCnodes, vx, vy, vz, l->locations);
    else
        launchDependent(bcPostKernel<S, KIND, false>, blocks, 128, 0, stream, dist, lat,
                        l->k, q, l->numberOfBCnodes, vx, vy, vz, l->locations);
}

template <class S>
static int launchPost(int kind, const vfb_bc_lattice* t, const vfb_bc_list* l, cudaStream_t stream)
{
    using R = typename Storage<S>::R;
    BcLattice<R> lat { t->numberOfLBnodes, t->neighborX, t->neighborY, t->neighborZ, (R)t->omega };
    S* dist = static_cast<S*>(t->distributions);
    const unsigned blocks = (l->numberOfBCnodes + 127) / 128;
    const bool even = t->isEvenTimestep != 0;
    switch (kind) {
    case VFB_BC_NOSLIP_INTERPOLATED: launchPostKind<S, VFB_BC_NOSLIP_INTERPOLATED>(even, blocks, stream, dist, lat, l); break;
    case VFB_BC_NOSLIP_BOUNCE_BACK: launchPostKind<S, VFB_BC_NOSLIP_BOUNCE_BACK>(even, blocks, stream, dist, lat, l); break;
    case VFB_BC_VELOCITY_INTERPOLATED: launchPostKind<S, VFB_BC_VELOCITY_INTERPOLATED>(even, blocks, stream, dist, lat, l); break;
    case VFB_BC_VELOCITY_BOUNCE_BACK: launchPostKind<S, VFB_BC_VELOCITY_BOUNCE_BACK>(even, blocks, stream, dist, lat, l); break;
    case VFB_BC_VELOCITY_WITH_PRESSURE:
        launchPostKind<S, VFB_BC_VELOCITY_WITH_PRESSURE>(even, blocks, stream, dist, lat, l);
        break;
    default: launchPostKind<S, VFB_BC_SLIP>(even, blocks, stream, dist, lat, l); break;
    }
    return checkLaunch("post-collision boundary condition");
}

template <class S>
static int launchPressure(const vfb_bc_lattice* t, const int32_t* k, const int32_t* kN, const void* rhoBC, uint32_t n,
                          int axis, int sgn, cudaStream_t stream, const uint32_t* locations = nullptr)
{
    using R = typename Storage<S>::R;
    BcLattice<R> lat { t->numberOfLBnodes, t->neighborX, t->neighborY, t->neighborZ, (R)t->omega };
    S* dist = static_cast<S*>(t->distributions);
    const unsigned blocks = (n + 127) / 128;
    const R* rho = static_cast<const R*>(rhoBC);
    if (t->isEvenTimestep)
        launchDependent(bcPressureKernel<S, true>, blocks, 128, 0, stream, dist, lat, k, kN, rho, n, axis, sgn,
                        locations);
    else
        launchDependent(bcPressureKernel<S, false>, blocks, 128, 0, stream, dist, lat, k, kN, rho, n, axis, sgn,
                        locations);
    return checkLaunch("pressure boundary condition");
}

template <class S>
static int launchOutflow(const vfb_bc_lattice* t, const int32_t* k, const int32_t* kN, uint32_t n, int axis, int sgn,
                         bool correction, double factor, cudaStream_t stream)
{
    using R = typename Storage<S>::R;
    BcLattice<R> lat { t->numberOfLBnodes, t->neighborX, t->neighborY, t->neighborZ, (R)t->omega };
    S* dist = static_cast<S*>(t->distributions);
    const unsigned blocks = (n + 127) / 128;
    // cs = 1 / sqrtf(3): the reference takes a single-precision root in both precisions
    const R cs = R(1) / R(std::sqrt(3.0f));
    const R fac = (R)factor;
    const bool even = t->isEvenTimestep != 0;
    if (correction) {
        if (even)
            launchDependent(bcOutflowKernel<S, true, true>, blocks, 128, 0, stream, dist, lat, k, kN, n, axis, sgn, cs,
                            fac);
        else
            launchDependent(bcOutflowKernel<S, false, true>, blocks, 128, 0, stream, dist, lat, k, kN, n, axis, sgn, cs,
                            fac);
    } else {
        if (even)
            launchDependent(bcOutflowKernel<S, true, false>, blocks, 128, 0, stream, dist, lat, k, kN, n, axis, sgn, cs,
                            fac);
        else
            launchDependent(bcOutflowKernel<S, false, false>, blocks, 128, 0, stream, dist, lat, k, kN, n, axis, sgn,
                            cs, fac);
    }
    return checkLaunch("outflow boundary condition");
}

static int checkLattice(const vfb_bc_lattice* t)
{
    if (!t || !t->distributions || !t->neighborX || !t->neighborY || !t->neighborZ)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL lattice or lattice array");
    if (t->numberOfLBnodes < 2)
        return setError(VFB_ERR_OUT_OF_RANGE, "numberOfLBnodes %llu < 2", t->numberOfLBnodes);
    return VFB_OK;
}

} // namespace vfb

using namespace vfb;

extern "C" int vfb_bc_post(int kind, int storage, const vfb_bc_lattice* lattice, const vfb_bc_list* list, void* stream)
{
    clearError();
    if (kind < VFB_BC_NOSLIP_INTERPOLATED || kind > VFB_BC_VELOCITY_WITH_PRESSURE)
        return setError(VFB_ERR_INVALID_ARGUMENT, "unknown BC kind %d", kind);
    if (vfb_storage_bytes(storage) == 0)
        return setError(VFB_ERR_INVALID_ARGUMENT, "unknown storage %d", storage);
    if (!list)
        return setError(VFB_ERR_INVALID_ARGUMENT, "list is NULL");
    if (list->numberOfBCnodes == 0)
        return VFB_OK;
    if (const int rc = checkLattice(lattice))
        return rc;
    if (!list->k || !list->q)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL k or q of the BC list");
    if ((kind == VFB_BC_VELOCITY_INTERPOLATED || kind == VFB_BC_VELOCITY_BOUNCE_BACK ||
         kind == VFB_BC_VELOCITY_WITH_PRESSURE) &&
        (!list->Vx || !list->Vy || !list->Vz))
        return setError(VFB_ERR_INVALID_ARGUMENT, "velocity BC needs Vx, Vy, Vz");
    if ((kind == VFB_BC_NOSLIP_INTERPOLATED || kind == VFB_BC_VELOCITY_INTERPOLATED || kind == VFB_BC_SLIP ||
         kind == VFB_BC_VELOCITY_WITH_PRESSURE) &&
        !(lattice->omega > 0.0 && lattice->omega < 2.0 && lattice->omega != 1.0))
        return setError(VFB_ERR_INVALID_ARGUMENT, "omega %g outside (0, 2) or equal to 1 (the interpolation divides by 1 - omega)",
                        lattice->omega);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (storage) {
    case VFB_FP32: return launchPost<float>(kind, lattice, list, s);
    case VFB_FP64: return launchPost<double>(kind, lattice, list, s);
    case VFB_FP16: return launchPost<__half>(kind, lattice, list, s);
    case VFB_FX16: return launchPost<int16_t>(kind, lattice, list, s);
    case VFB_FX16W: return launchPost<fx16w_t>(kind, lattice, list, s);
    default: return launchPost<__nv_bfloat16>(kind, lattice, list, s);
    }
}

extern "C" int vfb_bc_locations(const int32_t* k, uint32_t numberOfBCnodes, const uint32_t* neighborX,
                                const uint32_t* neighborY, const uint32_t* neighborZ, uint32_t* out, void* stream)
{
    clearError();
    if (numberOfBCnodes == 0)
        return VFB_OK;
    if (!k || !neighborX || !neighborY || !neighborZ || !out)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    bcLocationsKernel<<<(numberOfBCnodes + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        k, numberOfBCnodes, neighborX, neighborY, neighborZ, out);
    return checkLaunch("BC location table");
}

extern "C" int vfb_bc_pressure_noneq(int storage, const vfb_bc_lattice* lattice, const int32_t* k, const int32_t* kN,
                                     const void* rhoBC, uint32_t numberOfBCnodes, int direction, void* stream)
{
    clearError();
    if (vfb_storage_bytes(storage) == 0)
        return setError(VFB_ERR_INVALID_ARGUMENT, "unknown storage %d", storage);
    if (numberOfBCnodes == 0)
        return VFB_OK;
    if (const int rc = checkLattice(lattice))
        return rc;
    if (!k || !kN || !rhoBC)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL k, kN or rhoBC");
    if (direction < dP00 || direction > d00M)
        return setError(VFB_ERR_INVALID_ARGUMENT, "direction %d is not an axis direction (1..6)", direction);
    const int axis = cx(direction) != 0 ? 0 : cy(direction) != 0 ? 1 : 2;
    const int sgn = axis == 0 ? cx(direction) : axis == 1 ? cy(direction) : cz(direction);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (storage) {
    case VFB_FP32: return launchPressure<float>(lattice, k, kN, rhoBC, numberOfBCnodes, axis, sgn, s);
    case VFB_FP64: return launchPressure<double>(lattice, k, kN, rhoBC, numberOfBCnodes, axis, sgn, s);
    case VFB_FP16: return launchPressure<__half>(lattice, k, kN, rhoBC, numberOfBCnodes, axis, sgn, s);
    case VFB_FX16: return launchPressure<int16_t>(lattice, k, kN, rhoBC, numberOfBCnodes, axis, sgn, s);
    case VFB_FX16W: return launchPressure<fx16w_t>(lattice, k, kN, rhoBC, numberOfBCnodes, axis, sgn, s);
    default: return launchPressure<__nv_bfloat16>(lattice, k, kN, rhoBC, numberOfBCnodes, axis, sgn, s);
    }
}

namespace vfb
{
// vfb_bc_pressure_noneq with the list's location table (16 * numberOfBCnodes:
// the eight locations of each node k, then of its neighbour kN; the
// simulation builds it once per list)
int pressureNoneqWithLocations(int storage, const vfb_bc_lattice* lattice, const int32_t* k, const int32_t* kN,
                               const void* rhoBC, uint32_t numberOfBCnodes, int direction, const uint32_t* locations,
                               void* stream)
{
    clearError();
    if (vfb_storage_bytes(storage) == 0)
        return setError(VFB_ERR_INVALID_ARGUMENT, "unknown storage %d", storage);
    if (numberOfBCnodes == 0)
        return VFB_OK;
    if (const int rc = checkLattice(lattice))
        return rc;
    if (!k || !kN || !rhoBC)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL k, kN or rhoBC");
    if (direction < dP00 || direction > d00M)
        return setError(VFB_ERR_INVALID_ARGUMENT, "direction %d is not an axis direction (1..6)", direction);
    const int axis = cx(direction) != 0 ? 0 : cy(direction) != 0 ? 1 : 2;
    const int sgn = axis == 0 ? cx(direction) : axis == 1 ? cy(direction) : cz(direction);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (storage) {
    case VFB_FP32: return launchPressure<float>(lattice, k, kN, rhoBC, numberOfBCnodes, axis, sgn, s, locations);
    case VFB_FP64: return launchPressure<double>(lattice, k, kN, rhoBC, numberOfBCnodes, axis, sgn, s, locations);
    case VFB_FP16: return launchPressure<__half>(lattice, k, kN, rhoBC, numberOfBCnodes, axis, sgn, s, locations);
    case VFB_FX16: return launchPressure<int16_t>(lattice, k, kN, rhoBC, numberOfBCnodes, axis, sgn, s, locations);
    case VFB_FX16W: return launchPressure<fx16w_t>(lattice, k, kN, rhoBC, numberOfBCnodes, axis, sgn, s, locations);
    default: return launchPressure<__nv_bfloat16>(lattice, k, kN, rhoBC, numberOfBCnodes, axis, sgn, s, locations);
    }
}
} // namespace vfb

extern "C" int vfb_bc_outflow_nonreflecting(int storage, const vfb_bc_lattice* lattice, const int32_t* k,
                                            const int32_t* kN, uint32_t numberOfBCnodes, int direction,
                                            int pressureCorrection, double correctionFactor, void* stream)
{
    clearError();
    if (vfb_storage_bytes(storage) == 0)
        return setError(VFB_ERR_INVALID_ARGUMENT, "unknown storage %d", storage);
    if (numberOfBCnodes == 0)
        return VFB_OK;
    if (const int rc = checkLattice(lattice))
        return rc;
    if (!k || !kN)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL k or kN");
    if (direction < dP00 || direction > d00M)
        return setError(VFB_ERR_INVALID_ARGUMENT, "direction %d is not an axis direction (1..6)", direction);
    if (!std::isfinite(correctionFactor))
        return setError(VFB_ERR_INVALID_ARGUMENT, "correction factor is not finite");
    const int axis = cx(direction) != 0 ? 0 : cy(direction) != 0 ? 1 : 2;
    const int sgn = axis == 0 ? cx(direction) : axis == 1 ? cy(direction) : cz(direction);
    const bool corr = pressureCorrection != 0;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (storage) {
    case VFB_FP32: return launchOutflow<float>(lattice, k, kN, numberOfBCnodes, axis, sgn, corr, correctionFactor, s);
    case VFB_FP64: return launchOutflow<double>(lattice, k, kN, numberOfBCnodes, axis, sgn, corr, correctionFactor, s);
    case VFB_FP16: return launchOutflow<__half>(lattice, k, kN, numberOfBCnodes, axis, sgn, corr, correctionFactor, s);
    case VFB_FX16: return launchOutflow<int16_t>(lattice, k, kN, numberOfBCnodes, axis, sgn, corr, correctionFactor, s);
    case VFB_FX16W: return launchOutflow<fx16w_t>(lattice, k, kN, numberOfBCnodes, axis, sgn, corr, correctionFactor, s);
    default:
        return launchOutflow<__nv_bfloat16>(lattice, k, kN, numberOfBCnodes, axis, sgn, corr, correctionFactor, s);
    }
}
