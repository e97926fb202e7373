// ref_gpu_device.cu -- launchers for the reference's own GPU kernels, compiled
// unmodified by nvcc for sm_100a.
//
// TEST INFRASTRUCTURE ONLY (oracle).  oracle/Makefile (target `refgpu`) compiles
// the reference's kernel sources where they lie, by include path, together with
// this file into _ref/libvfref_gpu_{f64,f32}.so.  The functions below launch
// those kernels exactly as the reference's host launchers do: 64 threads per
// block (Parameter.cpp:400) and the 2D grid of vf::cuda::getCudaGrid
// (cuda_helper/CudaGrid.cpp:49-62).  They serve as the same-device baseline
// ("the kernel to beat") and as a second parity anchor: the reference's own
// device code on the same GPU.
//
// PressureNonEquilibriumCompressible_Device is not launched from here: it calls
// __syncthreads() inside `if (nodeIndex < numberOfBCnodes)`
// (PressureNonEquilibriumCompressible.cu:70,174), a barrier under divergent
// control flow, so it is kept off the GPU.  Its parity stays anchored on the
// host build of the same source.
#include <cstdint>

#include <cuda_runtime.h>

#include <basics/DataTypes.h>
#include <lbm/collision/K17CompressibleNavierStokes.h>

#include "Calculation/Calculation.h"
#include "Utilities/KernelUtilities.h"
#include "Utilities/RunCollision.cuh"
#include "BoundaryConditions/NoSlip/NoSlip_Device.cuh"
#include "BoundaryConditions/Velocity/Velocity_Device.cuh"
#include "BoundaryConditions/Slip/Slip_Device.cuh"
#include "Kernel/Compressible/NavierStokes/B92/B92CompressibleNavierStokes_Device.cuh"

template <bool b>
__global__ void scaleCoarseToFineCompressible_Device(real*, real*, unsigned int*, unsigned int*, unsigned int*,
                                                     unsigned int*, unsigned int*, unsigned int*, unsigned long long,
                                                     unsigned long long, bool, unsigned int*, unsigned int*,
                                                     unsigned int, real, real, real*, real*, ICellNeigh);
template <bool b>
__global__ void scaleFineToCoarseCompressible_Device(real*, real*, unsigned int*, unsigned int*, unsigned int*,
                                                     unsigned int*, unsigned int*, unsigned int*, unsigned long long,
                                                     unsigned long long, bool, unsigned int*, unsigned int*,
                                                     unsigned int, real, real, real*, real*, ICellNeigh);

// EnstrophyAnalyzer.cu:101-110 (the kernel; the file is compiled unmodified)
__global__ void enstrophyKernel(real* veloX, real* veloY, real* veloZ, real* rho, uint* neighborX, uint* neighborY,
                                uint* neighborZ, uint* neighborWSB, uint* geo, real* enstrophy, uint* isFluid,
                                unsigned long long numberOfLBnodes);

namespace
{
constexpr unsigned kThreads = 64; // Parameter.cpp:400 (numberofthreads)

// the launch grid of vf::cuda::getCudaGrid (CudaGrid.cpp:49-62): entities / threads + 1
// blocks, folded into rows of 512 once there are more than 512
dim3 referenceGrid(unsigned entities)
{
    const unsigned blocks = entities / kThreads + 1;
    if (blocks > 512)
        return dim3(512, blocks / 512 + 1);
    return dim3(1, blocks);
}

struct K17Functor {
    __device__ void operator()(vf::lbm::CollisionParameter& p, vf::lbm::MacroscopicValues& m,
                               vf::lbm::TurbulentViscosity& t) const
    {
        vf::lbm::runK17CompressibleNavierStokes<vf::lbm::TurbulenceModel::None>(p, m, t);
    }
};

inline cudaStream_t asStream(void* s) { return static_cast<cudaStream_t>(s); }
} // namespace

#ifdef VF_DOUBLE_ACCURACY
#define REF(name) name##_f64
#else
#define REF(name) name##_f32
#endif

extern "C" {

// K17CompressibleNavierStokes::runOnIndices, CollisionTemplate::Default
// (K17CompressibleNavierStokes.cu:117-124): runCollision<K17, None, false, false>
// over the fluid list, grid sized by the node count N (:155).  forces and
// limiters are device arrays of three values.
int REF(vfref_gpu_collision_k17)(real* dist, unsigned long long N, unsigned* nx, unsigned* ny, unsigned* nz,
                                 const unsigned* fluidNodes, unsigned nFluid, real omega, real* forces,
                                 real forceFactor, real* limiters, int isEven, void* stream)
{
    vf::gpu::GPUCollisionParameter p { omega,   nx,      ny,      nz,          dist,     nullptr, nullptr,
                                       nullptr, nullptr, nullptr, 0,           (int)N,   forceFactor, forces,
                                       nullptr, nullptr, nullptr, limiters,    isEven != 0, fluidNodes, nFluid };
    vf::gpu::runCollision<K17Functor, vf::lbm::TurbulenceModel::None, false, false>
        <<<referenceGrid((unsigned)N), kThreads, 0, asStream(stream)>>>(K17Functor {}, p);
    return (int)cudaGetLastError();
}

// B92CompressibleNavierStokes::run (B92CompressibleNavierStokes.cu:43-57): all N nodes
int REF(vfref_gpu_collision_bgk)(real* dist, unsigned long long N, unsigned* geo, unsigned* nx, unsigned* ny,
                                 unsigned* nz, real omega, int isEven, void* stream)
{
    B92CompressibleNavierStokes_Device<<<referenceGrid((unsigned)N), kThreads, 0, asStream(stream)>>>(
        omega, geo, nx, ny, nz, dist, (int)N, isEven != 0);
    return (int)cudaGetLastError();
}

// post-collision BC launchers (NoSlip.cu:81-98, Velocity.cu, Slip.cu); kind:
// 0 no-slip interpolated, 1 no-slip bounce-back, 2 velocity interpolated,
// 3 velocity bounce-back, 4 slip, 5 velocity with pressure interpolated.
// Returns -1 for another kind.
int REF(vfref_gpu_bc_post)(int kind, real* dist, unsigned long long N, unsigned* nx, unsigned* ny, unsigned* nz,
                           int* bcNodes, real* q, unsigned nBC, real omega, real* Vx, real* Vy, real* Vz, int isEven,
                           void* stream)
{
    const dim3 grid = referenceGrid(nBC);
    cudaStream_t s = asStream(stream);
    const bool ev = isEven != 0;
    switch (kind) {
    case 0: NoSlipInterpolatedCompressible_Device<<<grid, kThreads, 0, s>>>(dist, bcNodes, q, nBC, omega, nx, ny, nz, N, ev); break;
    case 1: NoSlipBounceBack_Device<<<grid, kThreads, 0, s>>>(dist, bcNodes, q, nBC, nx, ny, nz, N, ev); break;
    case 2:
        VelocityInterpolatedCompressible_Device<<<grid, kThreads, 0, s>>>(Vx, Vy, Vz, dist, bcNodes, q, nBC, omega, nx,
                                                                           ny, nz, N, ev);
        break;
    case 3: VelocityBounceBack_Device<<<grid, kThreads, 0, s>>>(Vx, Vy, Vz, dist, bcNodes, q, nBC, nx, ny, nz, N, ev); break;
    case 4: SlipCompressible_Device<<<grid, kThreads, 0, s>>>(dist, bcNodes, q, nBC, omega, nx, ny, nz, N, ev); break;
    case 5:
        VelocityWithPressureInterpolatedCompressible_Device<<<grid, kThreads, 0, s>>>(Vx, Vy, Vz, dist, bcNodes, q, nBC,
                                                                                       omega, nx, ny, nz, N, ev);
        break;
    default: return -1;
    }
    return (int)cudaGetLastError();
}

// scaleCoarseToFineCompressible<false> / scaleFineToCoarseCompressible<false>
// (Scaling.cu:105-180): one thread per interface cell, offsets as device arrays
int REF(vfref_gpu_scale_cf)(real* distC, real* distF, unsigned* nxC, unsigned* nyC, unsigned* nzC, unsigned* nxF,
                            unsigned* nyF, unsigned* nzF, unsigned long long NC, unsigned long long NF, int isEven,
                            unsigned* coarseCells, unsigned* fineCells, unsigned nCells, real omegaC, real omegaF,
                            real* offX, real* offY, real* offZ, void* stream)
{
    ICellNeigh off { offX, offY, offZ };
    scaleCoarseToFineCompressible_Device<false><<<referenceGrid(nCells), kThreads, 0, asStream(stream)>>>(
        distC, distF, nxC, nyC, nzC, nxF, nyF, nzF, NC, NF, isEven != 0, coarseCells, fineCells, nCells, omegaC,
        omegaF, nullptr, nullptr, off);
    return (int)cudaGetLastError();
}

int REF(vfref_gpu_scale_fc)(real* distC, real* distF, unsigned* nxC, unsigned* nyC, unsigned* nzC, unsigned* nxF,
                            unsigned* nyF, unsigned* nzF, unsigned long long NC, unsigned long long NF, int isEven,
                            unsigned* coarseCells, unsigned* fineCells, unsigned nCells, real omegaC, real omegaF,
                            real* offX, real* offY, real* offZ, void* stream)
{
    ICellNeigh off { offX, offY, offZ };
    scaleFineToCoarseCompressible_Device<false><<<referenceGrid(nCells), kThreads, 0, asStream(stream)>>>(
        distC, distF, nxC, nyC, nzC, nxF, nyF, nzF, NC, NF, isEven != 0, coarseCells, fineCells, nCells, omegaC,
        omegaF, nullptr, nullptr, off);
    return (int)cudaGetLastError();
}

// the kernel of EnstrophyAnalyzer::run (EnstrophyAnalyzer.cu:69-82): per node its
// enstrophy term and fluid flag into the zero-initialised arrays enstrophy and
// isFluid, one thread per node, launched as CudaGrid(numberofthreads, N) sizes it
int REF(vfref_gpu_enstrophy)(real* vx, real* vy, real* vz, real* rho, unsigned* nx, unsigned* ny, unsigned* nz,
                              unsigned* nNeg, unsigned* geo, real* enstrophy, unsigned* isFluid, unsigned long long N,
                              void* stream)
{
    enstrophyKernel<<<referenceGrid((unsigned)N), kThreads, 0, asStream(stream)>>>(vx, vy, vz, rho, nx, ny, nz, nNeg,
                                                                                   geo, enstrophy, isFluid, N);
    return (int)cudaGetLastError();
}

} // extern "C"
