// scaling.cu -- refinement-interface kernels: coarse-to-fine and
// fine-to-coarse interpolation (scaleCoarseToFineCompressible_Device,
// src/gpu/core/GridScaling/scaleCoarseToFineCompressible.cu:46-528;
// scaleFineToCoarseCompressible_Device, scaleFineToCoarseCompressible.cu:43-124;
// source moments gathered as in src/gpu/core/Utilities/ScalingUtilities.h:53-241).
//
// One thread per interface cell.  A cell is a 2x2x2 block of source nodes
// given by its base (most negative) node; the 27 nodes of the 3x3x3 block
// starting there hold the eight locations of each of the cell's nodes.  The
// block is walked through the neighbour arrays along the same paths as the
// reference (which matters only next to stoppers, where paths differ).
//   coarse to fine: moments of the 8 coarse nodes (pre-collision view of the
//     coarse parity) -> polynomial -> the 8 fine nodes at +-1/4 coarse
//     spacing, written into the fine pre-collision view of parity "even"
//     (the reference hard-wires the fine parity, scaleCoarseToFineCompressible.cu:59);
//   fine to coarse: moments of the 8 fine nodes (view "even",
//     scaleFineToCoarseCompressible.cu:105) -> polynomial -> the one coarse
//     node at the cell centre, written into the coarse pre-collision view.
// Coarse-to-fine cells of a real grid may write the same memory: cells repeat
// across periodic seams, and cells at the edge of the fine grid write stopper
// nodes whose locations alias those of other nodes.  The reference's kernel
// races there; its result applied cell by cell (cells in list order, corners
// in its visiting order) is made exact here by a write mask per cell and
// direction (vfb_scaling_write_mask) that leaves each memory cell to its last
// writer.  The fine-to-coarse cells of a grid write distinct coarse nodes.
#include <cuda_runtime.h>

#include <algorithm>

#include <unordered_map>
#include <vector>

#include "capi_common.cuh"
#include "d3q27.cuh"
#include "interpolation.cuh"
#include "storage.cuh"
#include "pdl.cuh"

namespace vfb
{

// the 3x3x3 block of sparse indices above a base node, B[x + 3 y + 9 z],
// along the reference's neighbour paths
__host__ __device__ __forceinline__ void blockWalk(uint32_t b, const uint32_t* nX, const uint32_t* nY,
                                                   const uint32_t* nZ, uint32_t* B)
{
#define VFB_B(x, y, z) B[(x) + 3 * (y) + 9 * (z)]
    VFB_B(0, 0, 0) = b;
    VFB_B(1, 0, 0) = nX[VFB_B(0, 0, 0)];
    VFB_B(0, 1, 0) = nY[VFB_B(0, 0, 0)];
    VFB_B(0, 0, 1) = nZ[VFB_B(0, 0, 0)];
    VFB_B(1, 1, 0) = nY[VFB_B(1, 0, 0)];
    VFB_B(1, 0, 1) = nZ[VFB_B(1, 0, 0)];
    VFB_B(0, 1, 1) = nZ[VFB_B(0, 1, 0)];
    VFB_B(1, 1, 1) = nZ[VFB_B(1, 1, 0)];
    VFB_B(0, 0, 2) = nZ[VFB_B(0, 0, 1)];
    VFB_B(1, 0, 2) = nZ[VFB_B(1, 0, 1)];
    VFB_B(0, 1, 2) = nZ[VFB_B(0, 1, 1)];
    VFB_B(1, 1, 2) = nZ[VFB_B(1, 1, 1)];
    VFB_B(2, 0, 1) = nX[VFB_B(1, 0, 1)];
    VFB_B(2, 1, 1) = nX[VFB_B(1, 1, 1)];
    VFB_B(2, 0, 2) = nX[VFB_B(1, 0, 2)];
    VFB_B(2, 1, 2) = nX[VFB_B(1, 1, 2)];
    VFB_B(2, 0, 0) = nX[VFB_B(1, 0, 0)];
    VFB_B(2, 1, 0) = nX[VFB_B(1, 1, 0)];
    VFB_B(0, 2, 0) = nY[VFB_B(0, 1, 0)];
    VFB_B(1, 2, 0) = nY[VFB_B(1, 1, 0)];
    VFB_B(0, 2, 1) = nY[VFB_B(0, 1, 1)];
    VFB_B(1, 2, 1) = nY[VFB_B(1, 1, 1)];
    VFB_B(0, 2, 2) = nZ[VFB_B(0, 2, 1)];
    VFB_B(1, 2, 2) = nZ[VFB_B(1, 2, 1)];
    VFB_B(2, 2, 1) = nX[VFB_B(1, 2, 1)];
    VFB_B(2, 2, 2) = nX[VFB_B(1, 2, 2)];
    VFB_B(2, 2, 0) = nX[VFB_B(1, 2, 0)];
#undef VFB_B
}

// the order in which the reference's coarse-to-fine kernel visits the fine
// corners (MMM, MMP, PMP, PMM, MPM, MPP, PPP, PPM; corner bits x | y << 1 | z << 2)
__host__ __device__ constexpr int cfCornerOrder(int j)
{
    constexpr int t[8] = { 0, 4, 5, 1, 2, 6, 7, 3 };
    return t[j];
}

// location l (bit 0 x, 1 y, 2 z) of the cell node at corner c (same bits)
__host__ __device__ __forceinline__ uint32_t cornerLocation(const uint32_t* B, int c, int l)
{
    const int x = (c & 1) + (l & 1), y = ((c >> 1) & 1) + ((l >> 1) & 1), z = ((c >> 2) & 1) + ((l >> 2) & 1);
    return B[x + 3 * y + 9 * z];
}

// memory access of the one-thread cell functions (the host form: FP32 / FP64)
template <class S>
struct HostAccess {
    using R = S;
    static R load(const S* p, int) { return *p; }
    static void store(S* p, R v, int) { *p = v; }
};

template <class S, class R>
struct ScalingView {
    S* distC;
    S* distF;
    const uint32_t* nXc;
    const uint32_t* nYc;
    const uint32_t* nZc;
    const uint32_t* nXf;
    const uint32_t* nYf;
    const uint32_t* nZf;
    unsigned long long NC, NF;
    const uint32_t* coarseCells;
    const uint32_t* fineCells;
    uint32_t nCells;
    R omegaC, omegaF;
    const R* offX;
    const R* offY;
    const R* offZ;
    const uint8_t* mask; // coarse to fine: mask[27 i + d] bit c = corner c writes direction d (NULL: all)
    const uint32_t* blocksC; // the cells' coarse / fine blocks, 27 per cell (NULL: walk)
    const uint32_t* blocksF;
};

// the moments of the 8 source nodes of a cell (pre-collision view of parity EVEN);
// the corner loops here and in coarseToFineCell are unrolled so that the
// cell's node indices and the corner moment sets stay in registers
template <class A, bool EVEN, class S, class R>
__host__ __device__ __forceinline__ void cellSourceMoments(const S* dist, unsigned long long N, const uint32_t* B,
                                                           R omega, SourceMoments<R>* src)
{
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        R f[27];
#pragma unroll
        for (int d = 0; d < 27; ++d)
            f[d] = A::load(dist + (unsigned long long)slot<EVEN>(d) * N + cornerLocation(B, c, loc(d)), d);
        src[c] = sourceMoments(f, omega);
    }
}

template <class A, bool EVEN_C, class S, class R>
__host__ __device__ __forceinline__ void coarseToFineCell(const ScalingView<S, R>& v, uint32_t i)
{
    uint32_t B[27];
    blockWalk(v.coarseCells[i], v.nXc, v.nYc, v.nZc, B);
    SourceMoments<R> src[8];
    cellSourceMoments<A, EVEN_C>(v.distC, v.NC, B, v.omegaC, src);
    const InterpCoeffs<R> k = interpolationCoefficients(src, v.offX[i], v.offY[i], v.offZ[i]);
    blockWalk(v.fineCells[i], v.nXf, v.nYf, v.nZf, B);
    const uint8_t* writes = v.mask ? v.mask + 27 * (size_t)i : nullptr;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int c = cfCornerOrder(j);
        const R x = (c & 1) ? R(1) / R(4) : -R(1) / R(4);
        const R y = (c & 2) ? R(1) / R(4) : -R(1) / R(4);
        const R z = (c & 4) ? R(1) / R(4) : -R(1) / R(4);
        R f[27];
        interpolateCoarseToFine(f, k, v.omegaF, x, y, z);
#pragma unroll
        for (int d = 0; d < 27; ++d)
            if (!writes || ((writes[d] >> c) & 1))
                A::store(v.distF + (unsigned long long)slot<true>(d) * v.NF + cornerLocation(B, c, loc(d)), f[d], d);
    }
}

template <class A, bool EVEN_C, class S, class R>
__host__ __device__ __forceinline__ void fineToCoarseCell(const ScalingView<S, R>& v, uint32_t i)
{
    uint32_t B[27];
    blockWalk(v.fineCells[i], v.nXf, v.nYf, v.nZf, B);
    SourceMoments<R> src[8];
    cellSourceMoments<A, true>(v.distF, v.NF, B, v.omegaF, src);
    const InterpCoeffs<R> k = interpolationCoefficients(src, v.offX[i], v.offY[i], v.offZ[i]);
    R f[27];
    interpolateFineToCoarse(f, k, v.omegaC);
    // the coarse node's own eight locations
    const uint32_t kc = v.coarseCells[i];
    uint32_t L[8];
    L[0] = kc;
    L[1] = v.nXc[kc];
    L[2] = v.nYc[kc];
    L[4] = v.nZc[kc];
    L[3] = v.nYc[L[1]];
    L[5] = v.nZc[L[1]];
    L[6] = v.nZc[L[2]];
    L[7] = v.nZc[L[3]];
#pragma unroll
    for (int d = 0; d < 27; ++d)
        A::store(v.distC + (unsigned long long)slot<EVEN_C>(d) * v.NC + L[loc(d)], f[d], d);
}

// The device kernels give each cell eight threads (lanes 8g .. 8g + 7 of a
// warp, corner c = lane % 8): each thread walks the cell's block, loads the
// 27 populations of its own source corner and forms that corner's moments;
// the group gathers the eight moment sets with shuffles, every thread forms
// the same coefficients (interpolationCoefficients on the same eight sets, so
// the same values as the one-thread cell functions above), and the writes
// are shared out: fine corner c (coarse to fine) or the coarse node's
// directions d with d % 8 == c (fine to coarse).  Eight times the threads of
// a cell per cell keep eight times the loads in flight.
constexpr int kScalingThreads = 128; // 16 cells per block

// the eight corners' moments of the group of this lane, from each lane's own
template <class R>
__device__ __forceinline__ void gatherMoments(const SourceMoments<R>& mine, SourceMoments<R>* src)
{
    const int base = (int)(threadIdx.x & 31u) & ~7;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        src[c].drho = __shfl_sync(0xffffffffu, mine.drho, base + c);
        src[c].vx = __shfl_sync(0xffffffffu, mine.vx, base + c);
        src[c].vy = __shfl_sync(0xffffffffu, mine.vy, base + c);
        src[c].vz = __shfl_sync(0xffffffffu, mine.vz, base + c);
        src[c].kxy = __shfl_sync(0xffffffffu, mine.kxy, base + c);
        src[c].kyz = __shfl_sync(0xffffffffu, mine.kyz, base + c);
        src[c].kxz = __shfl_sync(0xffffffffu, mine.kxz, base + c);
        src[c].kxxMyy = __shfl_sync(0xffffffffu, mine.kxxMyy, base + c);
        src[c].kxxMzz = __shfl_sync(0xffffffffu, mine.kxxMzz, base + c);
    }
}

// the eight locations of corner c of a block (a switch over the lane's corner
// keeps every index into B a constant, so B stays in registers)
template <int C>
__device__ __forceinline__ void cornerLocationsOf(const uint32_t* B, uint32_t* Lc)
{
#pragma unroll
    for (int l = 0; l < 8; ++l)
        Lc[l] = cornerLocation(B, C, l);
}

__device__ __forceinline__ void cornerLocations(const uint32_t* B, int c, uint32_t* Lc)
{
    switch (c) {
    case 0: cornerLocationsOf<0>(B, Lc); break;
    case 1: cornerLocationsOf<1>(B, Lc); break;
    case 2: cornerLocationsOf<2>(B, Lc); break;
    case 3: cornerLocationsOf<3>(B, Lc); break;
    case 4: cornerLocationsOf<4>(B, Lc); break;
    case 5: cornerLocationsOf<5>(B, Lc); break;
    case 6: cornerLocationsOf<6>(B, Lc); break;
    default: cornerLocationsOf<7>(B, Lc); break;
    }
}

// the eight locations of corner c of cell i: from the cell's block table
// (eight independent loads) or by walking the neighbour arrays
__device__ __forceinline__ void cellCornerLocations(const uint32_t* __restrict__ blocks, const uint32_t* cells,
                                                    const uint32_t* nX, const uint32_t* nY, const uint32_t* nZ,
                                                    uint32_t i, int c, uint32_t* Lc)
{
    if (blocks) {
        const uint32_t* row = blocks + 27ull * i;
#pragma unroll
        for (int l = 0; l < 8; ++l) {
            const int x = (c & 1) + (l & 1), y = ((c >> 1) & 1) + ((l >> 1) & 1), z = ((c >> 2) & 1) + ((l >> 2) & 1);
            Lc[l] = __ldg(row + x + 3 * y + 9 * z);
        }
        return;
    }
    uint32_t B[27];
    blockWalk(cells[i], nX, nY, nZ, B);
    cornerLocations(B, c, Lc);
}

// the moments of the corner whose locations are Lc (pre-collision view of parity EVEN)
template <bool EVEN, class S, class R>
__device__ __forceinline__ SourceMoments<R> cornerMoments(const S* dist, unsigned long long N, const uint32_t* Lc, R omega)
{
    R f[27];
#pragma unroll
    for (int d = 0; d < 27; ++d)
        f[d] = Storage<S>::load(dist + (unsigned long long)slot<EVEN>(d) * N + Lc[loc(d)], d);
    return sourceMoments(f, omega);
}

// the cells of block `block` (16 cells, eight threads each)
template <class S, bool EVEN_C>
__device__ __forceinline__ void coarseToFineBlock(const ScalingView<S, typename Storage<S>::R>& v, uint32_t block)
{
    using R = typename Storage<S>::R;
    const uint32_t i = (block * blockDim.x + threadIdx.x) >> 3;
    const int c = (int)(threadIdx.x & 7u);
    const bool active = i < v.nCells;
    // every lane takes part in the shuffles: a group past the end works on the last cell
    const uint32_t ic = active ? i : v.nCells - 1;
    uint32_t Lc[8];
    cellCornerLocations(v.blocksC, v.coarseCells, v.nXc, v.nYc, v.nZc, ic, c, Lc);
    SourceMoments<R> src[8];
    gatherMoments(cornerMoments<EVEN_C>(v.distC, v.NC, Lc, v.omegaC), src);
    const InterpCoeffs<R> k = interpolationCoefficients(src, v.offX[ic], v.offY[ic], v.offZ[ic]);
    if (!active)
        return;
    cellCornerLocations(v.blocksF, v.fineCells, v.nXf, v.nYf, v.nZf, ic, c, Lc);
    const R x = (c & 1) ? R(1) / R(4) : -R(1) / R(4);
    const R y = (c & 2) ? R(1) / R(4) : -R(1) / R(4);
    const R z = (c & 4) ? R(1) / R(4) : -R(1) / R(4);
    R f[27];
    interpolateCoarseToFine(f, k, v.omegaF, x, y, z);
    const uint8_t* writes = v.mask ? v.mask + 27 * (size_t)ic : nullptr;
#pragma unroll
    for (int d = 0; d < 27; ++d)
        if (!writes || ((writes[d] >> c) & 1))
            Storage<S>::store(v.distF + (unsigned long long)slot<true>(d) * v.NF + Lc[loc(d)], f[d], d);
}

template <class S, bool EVEN_C>
__device__ __forceinline__ void fineToCoarseBlock(const ScalingView<S, typename Storage<S>::R>& v, uint32_t block)
{
    using R = typename Storage<S>::R;
    const uint32_t i = (block * blockDim.x + threadIdx.x) >> 3;
    const int c = (int)(threadIdx.x & 7u);
    const bool active = i < v.nCells;
    const uint32_t ic = active ? i : v.nCells - 1;
    uint32_t Lc[8];
    cellCornerLocations(v.blocksF, v.fineCells, v.nXf, v.nYf, v.nZf, ic, c, Lc);
    SourceMoments<R> src[8];
    gatherMoments(cornerMoments<true>(v.distF, v.NF, Lc, v.omegaF), src);
    const InterpCoeffs<R> k = interpolationCoefficients(src, v.offX[ic], v.offY[ic], v.offZ[ic]);
    if (!active)
        return;
    R f[27];
    interpolateFineToCoarse(f, k, v.omegaC);
    // the coarse node's own eight locations (corner 0 of its block)
    uint32_t L[8];
    cellCornerLocations(v.blocksC, v.coarseCells, v.nXc, v.nYc, v.nZc, ic, 0, L);
#pragma unroll
    for (int d = 0; d < 27; ++d)
        if ((d & 7) == c)
            Storage<S>::store(v.distC + (unsigned long long)slot<EVEN_C>(d) * v.NC + L[loc(d)], f[d], d);
}

template <class S, bool EVEN_C>
__global__ void __launch_bounds__(kScalingThreads) coarseToFineKernel(const ScalingView<S, typename Storage<S>::R> v)
{
    gridDependencyWait();
    coarseToFineBlock<S, EVEN_C>(v, blockIdx.x);
}

template <class S, bool EVEN_C>
__global__ void __launch_bounds__(kScalingThreads) fineToCoarseKernel(const ScalingView<S, typename Storage<S>::R> v)
{
    gridDependencyWait();
    fineToCoarseBlock<S, EVEN_C>(v, blockIdx.x);
}

// both lists of a level pair in one launch: the first fcBlocks blocks take
// the fine-to-coarse cells, the rest the coarse-to-fine cells (valid when
// neither list reads what the other writes, vfb_scaling_independent)
template <class S, bool EVEN_C>
__global__ void __launch_bounds__(kScalingThreads)
    interfaceKernel(const ScalingView<S, typename Storage<S>::R> fc, const ScalingView<S, typename Storage<S>::R> cf,
                    uint32_t fcBlocks)
{
    gridDependencyWait();
    if (blockIdx.x < fcBlocks)
        fineToCoarseBlock<S, EVEN_C>(fc, blockIdx.x);
    else
        coarseToFineBlock<S, EVEN_C>(cf, blockIdx.x - fcBlocks);
}

template <class S, class R>
static ScalingView<S, R> viewOf(const vfb_scaling_args* a)
{
    ScalingView<S, R> v;
    v.distC = static_cast<S*>(a->distributionsCoarse);
    v.distF = static_cast<S*>(a->distributionsFine);
    v.nXc = a->neighborXcoarse;
    v.nYc = a->neighborYcoarse;
    v.nZc = a->neighborZcoarse;
    v.nXf = a->neighborXfine;
    v.nYf = a->neighborYfine;
    v.nZf = a->neighborZfine;
    v.NC = a->numberOfLBnodesCoarse;
    v.NF = a->numberOfLBnodesFine;
    v.coarseCells = a->coarseCells;
    v.fineCells = a->fineCells;
    v.nCells = a->numberOfCells;
    v.omegaC = (R)a->omegaCoarse;
    v.omegaF = (R)a->omegaFine;
    v.offX = static_cast<const R*>(a->offsetX);
    v.offY = static_cast<const R*>(a->offsetY);
    v.offZ = static_cast<const R*>(a->offsetZ);
    v.mask = a->fineWriteMask;
    v.blocksC = a->coarseBlocks;
    v.blocksF = a->fineBlocks;
    return v;
}

template <class S>
static int launchScaling(bool cf, const vfb_scaling_args* a, cudaStream_t s)
{
    using R = typename Storage<S>::R;
    const ScalingView<S, R> v = viewOf<S, R>(a);
    if (a->numberOfCells == 0)
        return VFB_OK;
    constexpr unsigned cellsPerBlock = kScalingThreads / 8;
    const unsigned blocks = (a->numberOfCells + cellsPerBlock - 1) / cellsPerBlock;
    if (cf) {
        if (a->isEvenTimestep)
            launchDependent(coarseToFineKernel<S, true>, blocks, kScalingThreads, 0, s, v);
        else
            launchDependent(coarseToFineKernel<S, false>, blocks, kScalingThreads, 0, s, v);
    } else {
        if (a->isEvenTimestep)
            launchDependent(fineToCoarseKernel<S, true>, blocks, kScalingThreads, 0, s, v);
        else
            launchDependent(fineToCoarseKernel<S, false>, blocks, kScalingThreads, 0, s, v);
    }
    return checkLaunch(cf ? "coarse-to-fine interpolation" : "fine-to-coarse interpolation");
}

static int checkScalingArgs(int storage, const vfb_scaling_args* a)
{
    if (vfb_storage_bytes(storage) == 0)
        return setError(VFB_ERR_INVALID_ARGUMENT, "unknown storage %d", storage);
    if (!a)
        return setError(VFB_ERR_INVALID_ARGUMENT, "args is NULL");
    if (a->numberOfCells == 0)
        return VFB_OK;
    if (!a->distributionsCoarse || !a->distributionsFine || !a->neighborXcoarse || !a->neighborYcoarse ||
        !a->neighborZcoarse || !a->neighborXfine || !a->neighborYfine || !a->neighborZfine || !a->coarseCells ||
        !a->fineCells || !a->offsetX || !a->offsetY || !a->offsetZ)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL array in scaling args");
    if (!(a->omegaCoarse > 0.0 && a->omegaCoarse < 2.0 && a->omegaFine > 0.0 && a->omegaFine < 2.0))
        return setError(VFB_ERR_INVALID_ARGUMENT, "omega outside (0, 2)");
    return VFB_OK;
}

static int runScaling(bool cf, int storage, const vfb_scaling_args* a, void* stream)
{
    clearError();
    if (const int rc = checkScalingArgs(storage, a))
        return rc;
    if (a->numberOfCells == 0)
        return VFB_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (storage) {
    case VFB_FP32: return launchScaling<float>(cf, a, s);
    case VFB_FP64: return launchScaling<double>(cf, a, s);
    case VFB_FP16: return launchScaling<__half>(cf, a, s);
    case VFB_FX16: return launchScaling<int16_t>(cf, a, s);
    case VFB_FX16W: return launchScaling<fx16w_t>(cf, a, s);
    default: return launchScaling<__nv_bfloat16>(cf, a, s);
    }
}

template <class S>
static int launchInterface(const vfb_scaling_args* fc, const vfb_scaling_args* cf, cudaStream_t s)
{
    using R = typename Storage<S>::R;
    constexpr unsigned cellsPerBlock = kScalingThreads / 8;
    const unsigned fcBlocks = (fc->numberOfCells + cellsPerBlock - 1) / cellsPerBlock;
    const unsigned cfBlocks = (cf->numberOfCells + cellsPerBlock - 1) / cellsPerBlock;
    const ScalingView<S, R> vf = viewOf<S, R>(fc), vc = viewOf<S, R>(cf);
    if (fc->isEvenTimestep)
        launchDependent(interfaceKernel<S, true>, fcBlocks + cfBlocks, kScalingThreads, 0, s, vf, vc, fcBlocks);
    else
        launchDependent(interfaceKernel<S, false>, fcBlocks + cfBlocks, kScalingThreads, 0, s, vf, vc, fcBlocks);
    return checkLaunch("fine-to-coarse and coarse-to-fine interpolation");
}

template <class S>
static void hostScaling(bool cf, const vfb_scaling_args* a)
{
    const ScalingView<S, S> v = viewOf<S, S>(a);
    for (uint32_t i = 0; i < v.nCells; ++i) {
        if (cf)
            a->isEvenTimestep ? coarseToFineCell<HostAccess<S>, true>(v, i) : coarseToFineCell<HostAccess<S>, false>(v, i);
        else
            a->isEvenTimestep ? fineToCoarseCell<HostAccess<S>, true>(v, i) : fineToCoarseCell<HostAccess<S>, false>(v, i);
    }
}

} // namespace vfb

using namespace vfb;

extern "C" int vfb_scaling_write_mask(const uint32_t* fineCells, uint32_t n, const uint32_t* nXf, const uint32_t* nYf,
                                      const uint32_t* nZf, unsigned long long NF, uint8_t* mask)
{
    clearError();
    if (n == 0)
        return VFB_OK;
    if (!fineCells || !nXf || !nYf || !nZf || !mask || NF == 0)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    // the last write (cell order, then the reference's corner order) to each
    // memory cell (slot d of the even view, location index)
    std::unordered_map<unsigned long long, uint32_t> last;
    last.reserve((size_t)n * 216);
    std::vector<unsigned long long> target((size_t)n * 216);
    for (uint32_t i = 0; i < n; ++i) {
        if (fineCells[i] >= NF)
            return setError(VFB_ERR_OUT_OF_RANGE, "fine cell %u: base node %u outside the level", i, fineCells[i]);
        uint32_t B[27];
        blockWalk(fineCells[i], nXf, nYf, nZf, B);
        for (int b = 0; b < 27; ++b)
            if (B[b] >= NF)
                return setError(VFB_ERR_OUT_OF_RANGE, "fine cell %u: node %u outside the level", i, B[b]);
        for (int j = 0; j < 8; ++j) {
            const int c = cfCornerOrder(j);
            for (int d = 0; d < 27; ++d) {
                const unsigned long long cell = (unsigned long long)slot<true>(d) * NF + cornerLocation(B, c, loc(d));
                const size_t w = (size_t)i * 216 + (size_t)c * 27 + (size_t)d;
                target[w] = cell;
                last[cell] = (uint32_t)w;
            }
        }
    }
    for (uint32_t i = 0; i < n; ++i)
        for (int d = 0; d < 27; ++d) {
            uint8_t m = 0;
            for (int c = 0; c < 8; ++c) {
                const size_t w = (size_t)i * 216 + (size_t)c * 27 + (size_t)d;
                if (last[target[w]] == (uint32_t)w)
                    m |= (uint8_t)(1u << c);
            }
            mask[27 * (size_t)i + d] = m;
        }
    return VFB_OK;
}

extern "C" int vfb_scale_coarse_to_fine(int storage, const vfb_scaling_args* args, void* stream)
{
    return runScaling(true, storage, args, stream);
}

__global__ void scalingBlocksKernel(const uint32_t* __restrict__ cells, uint32_t n, const uint32_t* __restrict__ nX,
                                    const uint32_t* __restrict__ nY, const uint32_t* __restrict__ nZ,
                                    uint32_t* __restrict__ out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    uint32_t B[27];
    blockWalk(cells[i], nX, nY, nZ, B);
#pragma unroll
    for (int j = 0; j < 27; ++j)
        out[27ull * i + j] = B[j];
}

extern "C" int vfb_scaling_blocks(const uint32_t* cells, uint32_t n, const uint32_t* nX, const uint32_t* nY,
                                  const uint32_t* nZ, uint32_t* out, void* stream)
{
    clearError();
    if (n == 0)
        return VFB_OK;
    if (!cells || !nX || !nY || !nZ || !out)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    scalingBlocksKernel<<<(n + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(cells, n, nX, nY, nZ, out);
    return checkLaunch("interface cell blocks");
}

extern "C" int vfb_scale_interface(int storage, const vfb_scaling_args* fineToCoarse,
                                   const vfb_scaling_args* coarseToFine, void* stream)
{
    clearError();
    if (const int rc = checkScalingArgs(storage, fineToCoarse))
        return rc;
    if (const int rc = checkScalingArgs(storage, coarseToFine))
        return rc;
    if (fineToCoarse->isEvenTimestep != coarseToFine->isEvenTimestep)
        return setError(VFB_ERR_INVALID_ARGUMENT, "the two lists' parities differ");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (fineToCoarse->numberOfCells == 0 || coarseToFine->numberOfCells == 0) {
        if (const int rc = runScaling(false, storage, fineToCoarse, stream))
            return rc;
        return runScaling(true, storage, coarseToFine, stream);
    }
    switch (storage) {
    case VFB_FP32: return launchInterface<float>(fineToCoarse, coarseToFine, s);
    case VFB_FP64: return launchInterface<double>(fineToCoarse, coarseToFine, s);
    case VFB_FP16: return launchInterface<__half>(fineToCoarse, coarseToFine, s);
    case VFB_FX16: return launchInterface<int16_t>(fineToCoarse, coarseToFine, s);
    case VFB_FX16W: return launchInterface<fx16w_t>(fineToCoarse, coarseToFine, s);
    default: return launchInterface<__nv_bfloat16>(fineToCoarse, coarseToFine, s);
    }
}

extern "C" int vfb_scaling_independent(const uint32_t* fcCoarse, const uint32_t* fcFine, uint32_t nFC,
                                       const uint32_t* cfCoarse, const uint32_t* cfFine, uint32_t nCF,
                                       const uint8_t* cfMask, const uint32_t* nXc, const uint32_t* nYc,
                                       const uint32_t* nZc, unsigned long long NC, const uint32_t* nXf,
                                       const uint32_t* nYf, const uint32_t* nZf, unsigned long long NF,
                                       int* independent)
{
    clearError();
    if (!independent)
        return setError(VFB_ERR_INVALID_ARGUMENT, "independent is NULL");
    *independent = 0;
    if ((nFC && (!fcCoarse || !fcFine)) || (nCF && (!cfCoarse || !cfFine)) || !nXc || !nYc || !nZc || !nXf ||
        !nYf || !nZf || NC == 0 || NF == 0)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    auto inRange = [](uint32_t k, unsigned long long n) { return (unsigned long long)k < n; };
    uint32_t B[27];
    // fine side: the cells the coarse-to-fine list writes, against those the fine-to-coarse list reads
    std::vector<uint8_t> written(27ull * NF, 0);
    for (uint32_t i = 0; i < nCF; ++i) {
        if (!inRange(cfFine[i], NF))
            return setError(VFB_ERR_OUT_OF_RANGE, "coarse-to-fine cell %u: fine node outside the level", i);
        blockWalk(cfFine[i], nXf, nYf, nZf, B);
        for (int c = 0; c < 8; ++c)
            for (int d = 0; d < 27; ++d)
                if (!cfMask || ((cfMask[27ull * i + d] >> c) & 1))
                    written[(unsigned long long)slot<true>(d) * NF + cornerLocation(B, c, loc(d))] = 1;
    }
    for (uint32_t i = 0; i < nFC; ++i) {
        if (!inRange(fcFine[i], NF))
            return setError(VFB_ERR_OUT_OF_RANGE, "fine-to-coarse cell %u: fine node outside the level", i);
        blockWalk(fcFine[i], nXf, nYf, nZf, B);
        for (int c = 0; c < 8; ++c)
            for (int d = 0; d < 27; ++d)
                if (written[(unsigned long long)slot<true>(d) * NF + cornerLocation(B, c, loc(d))])
                    return VFB_OK;
    }
    // coarse side, both parities: the cells the fine-to-coarse list writes,
    // against those the coarse-to-fine list reads
    std::vector<uint8_t> wc(27ull * NC);
    for (int parity = 0; parity < 2; ++parity) {
        std::fill(wc.begin(), wc.end(), 0);
        for (uint32_t i = 0; i < nFC; ++i) {
            const uint32_t kc = fcCoarse[i];
            if (!inRange(kc, NC))
                return setError(VFB_ERR_OUT_OF_RANGE, "fine-to-coarse cell %u: coarse node outside the level", i);
            uint32_t L[8];
            L[0] = kc;
            L[1] = nXc[kc];
            L[2] = nYc[kc];
            L[4] = nZc[kc];
            L[3] = nYc[L[1]];
            L[5] = nZc[L[1]];
            L[6] = nZc[L[2]];
            L[7] = nZc[L[3]];
            for (int d = 0; d < 27; ++d)
                wc[(unsigned long long)(parity ? slot<true>(d) : slot<false>(d)) * NC + L[loc(d)]] = 1;
        }
        for (uint32_t i = 0; i < nCF; ++i) {
            if (!inRange(cfCoarse[i], NC))
                return setError(VFB_ERR_OUT_OF_RANGE, "coarse-to-fine cell %u: coarse node outside the level", i);
            blockWalk(cfCoarse[i], nXc, nYc, nZc, B);
            for (int c = 0; c < 8; ++c)
                for (int d = 0; d < 27; ++d)
                    if (wc[(unsigned long long)(parity ? slot<true>(d) : slot<false>(d)) * NC +
                           cornerLocation(B, c, loc(d))])
                        return VFB_OK;
        }
    }
    *independent = 1;
    return VFB_OK;
}

extern "C" int vfb_scale_fine_to_coarse(int storage, const vfb_scaling_args* args, void* stream)
{
    return runScaling(false, storage, args, stream);
}

extern "C" int vfb_debug_scale_host(int coarseToFine, int precision, const vfb_scaling_args* args)
{
    clearError();
    if (precision != VFB_FP32 && precision != VFB_FP64)
        return setError(VFB_ERR_INVALID_ARGUMENT, "precision must be VFB_FP32 or VFB_FP64");
    if (const int rc = checkScalingArgs(precision, args))
        return rc;
    if (precision == VFB_FP64)
        hostScaling<double>(coarseToFine != 0, args);
    else
        hostScaling<float>(coarseToFine != 0, args);
    return VFB_OK;
}
