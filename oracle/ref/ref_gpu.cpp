// ref_gpu.cpp -- harness around the reference's own GPU kernel sources.
//
// TEST INFRASTRUCTURE ONLY (oracle).  The reference kernels
// (src/gpu/core/.../*.cu) are compiled as plain host C++ by oracle/Makefile
// with the stand-in CUDA headers of oracle/stubs; every __global__ function
// then becomes an ordinary function.  The functions below emulate one kernel
// launch by calling that function once per thread index, sequentially, after
// setting the emulated thread coordinates so that
// vf::cuda::get1DIndexFrom2DBlock() (src/gpu/cuda_helper/CudaIndexCalculation.h:42)
// returns the index of the emulated thread.  The reference kernels do not
// communicate between threads, so the sequential emulation computes what one
// launch computes.
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
#include "BoundaryConditions/Pressure/Pressure_Device.cuh"
#include "BoundaryConditions/Outflow/Outflow_Device.cuh"
#include "BoundaryConditions/Stress/Stress_Device.cuh"
#include "Kernel/Compressible/NavierStokes/B92/B92CompressibleNavierStokes_Device.cuh"
#include "PreProcessor/PreProcessorStrategy/InitNavierStokesCompressible/InitNavierStokesCompressible_Device.cuh"

thread_local uint3 threadIdx;
thread_local uint3 blockIdx;
thread_local dim3 blockDim;
thread_local dim3 gridDim;

template <bool b>
void scaleCoarseToFineCompressible_Device(real*, real*, unsigned int*, unsigned int*, unsigned int*, unsigned int*,
                                          unsigned int*, unsigned int*, unsigned long long, unsigned long long, bool,
                                          unsigned int*, unsigned int*, unsigned int, real, real, real*, real*, ICellNeigh);
template <bool b>
void scaleFineToCoarseCompressible_Device(real*, real*, unsigned int*, unsigned int*, unsigned int*, unsigned int*,
                                          unsigned int*, unsigned int*, unsigned long long, unsigned long long, bool,
                                          unsigned int*, unsigned int*, unsigned int, real, real, real*, real*, ICellNeigh);

namespace
{
// thread t of the emulated launch: blockDim.x = 1, gridDim.x = 1, blockIdx.y = t
inline void setThread(unsigned long long t)
{
    blockDim = dim3(1, 1, 1);
    gridDim = dim3(1, 1, 1);
    threadIdx = uint3 { 0, 0, 0 };
    blockIdx = uint3 { 0, (unsigned)t, 0 };
}

struct K17Functor {
    void operator()(vf::lbm::CollisionParameter& p, vf::lbm::MacroscopicValues& m, vf::lbm::TurbulentViscosity& t) const
    {
        vf::lbm::runK17CompressibleNavierStokes<vf::lbm::TurbulenceModel::None>(p, m, t);
    }
};
} // namespace

#ifdef VF_DOUBLE_ACCURACY
#define REF(name) name##_f64
#else
#define REF(name) name##_f32
#endif

extern "C" {

// runCollision<K17, None, writeMacro, applyBodyForce> (RunCollision.cuh:74-143)
void REF(vfref_collision_k17)(real* dist, unsigned long long N, unsigned* nx, unsigned* ny, unsigned* nz,
                              const unsigned* fluidNodes, unsigned nFluid, real omega, real* forces, real forceFactor,
                              real* limiters, int isEven, int flags, real* rho, real* vx, real* vy, real* vz,
                              real* bfx, real* bfy, real* bfz)
{
    vf::gpu::GPUCollisionParameter p { omega, nx, ny, nz, dist, rho, vx, vy, vz, nullptr, 0, (int)N, forceFactor,
                                       forces, bfx, bfy, bfz, limiters, isEven != 0, fluidNodes, nFluid };
    K17Functor f;
    for (unsigned t = 0; t < nFluid; ++t) {
        setThread(t);
        switch (flags & 3) {
        case 0: vf::gpu::runCollision<K17Functor, vf::lbm::TurbulenceModel::None, false, false>(f, p); break;
        case 1: vf::gpu::runCollision<K17Functor, vf::lbm::TurbulenceModel::None, true, false>(f, p); break;
        case 2: vf::gpu::runCollision<K17Functor, vf::lbm::TurbulenceModel::None, false, true>(f, p); break;
        default: vf::gpu::runCollision<K17Functor, vf::lbm::TurbulenceModel::None, true, true>(f, p); break;
        }
    }
}

// B92CompressibleNavierStokes_Device over all nodes
void REF(vfref_collision_bgk)(real* dist, unsigned long long N, unsigned* geo, unsigned* nx, unsigned* ny,
                              unsigned* nz, real omega, int isEven)
{
    for (unsigned long long t = 0; t < N; ++t) {
        setThread(t);
        B92CompressibleNavierStokes_Device(omega, geo, nx, ny, nz, dist, (int)N, isEven != 0);
    }
}

// InitNavierStokesCompressible_Device for one parity
void REF(vfref_init_eq)(real* dist, unsigned long long N, unsigned* geo, unsigned* nx, unsigned* ny, unsigned* nz,
                        real* rho, real* ux, real* uy, real* uz, int isEven)
{
    for (unsigned long long t = 0; t < N; ++t) {
        setThread(t);
        InitNavierStokesCompressible_Device(nx, ny, nz, geo, rho, ux, uy, uz, (unsigned)N, dist, isEven != 0);
    }
}

// OutflowNonReflecting_Device (correction 0) or
// OutflowNonReflectingPressureCorrection_Device over one directional list
void REF(vfref_bc_outflow)(int correction, real* dist, unsigned long long N, unsigned* nx, unsigned* ny, unsigned* nz,
                           int* bcNodes, int* bcNeighbors, unsigned nBC, int direction, real factor, int isEven)
{
    for (unsigned t = 0; t < nBC; ++t) {
        setThread(t);
        if (correction)
            OutflowNonReflectingPressureCorrection_Device(nullptr, dist, bcNodes, bcNeighbors, (int)nBC, (real)1, nx, ny,
                                                          nz, N, isEven != 0, direction, factor);
        else
            OutflowNonReflecting_Device(nullptr, dist, bcNodes, bcNeighbors, (int)nBC, (real)1, nx, ny, nz, N,
                                        isEven != 0, direction);
    }
}

// InitNavierStokesCompressibleNonEquilibrium_Device for one parity
void REF(vfref_init_noneq)(real* dist, unsigned long long N, unsigned* geo, unsigned* nx, unsigned* ny, unsigned* nz,
                           unsigned* nneg, real* rho, real* ux, real* uy, real* uz, real omega, int isEven)
{
    for (unsigned long long t = 0; t < N; ++t) {
        setThread(t);
        InitNavierStokesCompressibleNonEquilibrium_Device(nx, ny, nz, nneg, geo, rho, ux, uy, uz, (unsigned)N, dist,
                                                          omega, isEven != 0);
    }
}

// post-collision BC kernels; kind: 0 no-slip interpolated, 1 no-slip
// bounce-back, 2 velocity interpolated, 3 velocity bounce-back, 4 slip,
// 5 velocity with pressure interpolated
void REF(vfref_bc_post)(int kind, real* dist, unsigned long long N, unsigned* nx, unsigned* ny, unsigned* nz,
                        int* bcNodes, real* q, unsigned nBC, real omega, real* Vx, real* Vy, real* Vz, int isEven)
{
    for (unsigned t = 0; t < nBC; ++t) {
        setThread(t);
        switch (kind) {
        case 0: NoSlipInterpolatedCompressible_Device(dist, bcNodes, q, nBC, omega, nx, ny, nz, N, isEven != 0); break;
        case 1: NoSlipBounceBack_Device(dist, bcNodes, q, nBC, nx, ny, nz, N, isEven != 0); break;
        case 2:
            VelocityInterpolatedCompressible_Device(Vx, Vy, Vz, dist, bcNodes, q, nBC, omega, nx, ny, nz, N, isEven != 0);
            break;
        case 3: VelocityBounceBack_Device(Vx, Vy, Vz, dist, bcNodes, q, nBC, nx, ny, nz, N, isEven != 0); break;
        case 4: SlipCompressible_Device(dist, bcNodes, q, nBC, omega, nx, ny, nz, N, isEven != 0); break;
        case 5:
            VelocityWithPressureInterpolatedCompressible_Device(Vx, Vy, Vz, dist, bcNodes, q, nBC, omega, nx, ny, nz, N,
                                                                isEven != 0);
            break;
        default: break;
        }
    }
}

// the wall-model (stress) kernels over one list; kind: 0 StressCompressible_Device,
// 1 StressBounceBackCompressible_Device, 2 StressBounceBackPressureCompressible_Device
// (Stress.cu:42-160 passes the level's velocityY as vz; the caller decides here)
void REF(vfref_bc_stress)(int kind, real* dist, unsigned long long N, unsigned* nx, unsigned* ny, unsigned* nz,
                          int* bcNodes, int* samplingNodes, real* q, unsigned nBC, real omega, real* turbViscosity,
                          real* vx, real* vy, real* vz, real* normalX, real* normalY, real* normalZ, real* vxEl,
                          real* vyEl, real* vzEl, real* vxWMean, real* vyWMean, real* vzWMean, int* samplingOffset,
                          real* z0, int hasMonitor, real* uStar, real* Fx, real* Fy, real* Fz, int isEven)
{
    for (unsigned t = 0; t < nBC; ++t) {
        setThread(t);
        switch (kind) {
        case 0:
            StressCompressible_Device(dist, bcNodes, samplingNodes, q, nBC, omega, turbViscosity, vx, vy, vz, normalX,
                                      normalY, normalZ, vxEl, vyEl, vzEl, vxWMean, vyWMean, vzWMean, samplingOffset, z0,
                                      hasMonitor != 0, uStar, Fx, Fy, Fz, nx, ny, nz, N, isEven != 0);
            break;
        case 1:
            StressBounceBackCompressible_Device(dist, bcNodes, samplingNodes, q, nBC, vx, vy, vz, normalX, normalY,
                                                normalZ, vxEl, vyEl, vzEl, vxWMean, vyWMean, vzWMean, samplingOffset,
                                                z0, hasMonitor != 0, uStar, Fx, Fy, Fz, nx, ny, nz, N, isEven != 0);
            break;
        default:
            StressBounceBackPressureCompressible_Device(dist, bcNodes, samplingNodes, q, nBC, vx, vy, vz, normalX,
                                                        normalY, normalZ, vxEl, vyEl, vzEl, vxWMean, vyWMean, vzWMean,
                                                        samplingOffset, z0, hasMonitor != 0, uStar, Fx, Fy, Fz, nx, ny,
                                                        nz, N, isEven != 0);
            break;
        }
    }
}

// PressureNonEquilibriumCompressible_Device for one directional list
void REF(vfref_bc_pressure_noneq)(real* dist, unsigned long long N, unsigned* nx, unsigned* ny, unsigned* nz,
                                  int* bcNodes, int* bcNeighbors, real* rhoBC, unsigned nBC, int direction, int isEven)
{
    for (unsigned t = 0; t < nBC; ++t) {
        setThread(t);
        PressureNonEquilibriumCompressible_Device(rhoBC, dist, bcNodes, bcNeighbors, (int)nBC, nx, ny, nz, N,
                                                  isEven != 0, (size_t)direction);
    }
}

// scaleCoarseToFineCompressible_Device<false> / scaleFineToCoarseCompressible_Device<false>
void REF(vfref_scale_cf)(real* distC, real* distF, unsigned* nxC, unsigned* nyC, unsigned* nzC, unsigned* nxF,
                         unsigned* nyF, unsigned* nzF, unsigned long long NC, unsigned long long NF, int isEven,
                         unsigned* coarseCells, unsigned* fineCells, unsigned nCells, real omegaC, real omegaF,
                         real* offX, real* offY, real* offZ)
{
    ICellNeigh off { offX, offY, offZ };
    for (unsigned t = 0; t < nCells; ++t) {
        setThread(t);
        scaleCoarseToFineCompressible_Device<false>(distC, distF, nxC, nyC, nzC, nxF, nyF, nzF, NC, NF, isEven != 0,
                                                    coarseCells, fineCells, nCells, omegaC, omegaF, nullptr, nullptr,
                                                    off);
    }
}

void REF(vfref_scale_fc)(real* distC, real* distF, unsigned* nxC, unsigned* nyC, unsigned* nzC, unsigned* nxF,
                         unsigned* nyF, unsigned* nzF, unsigned long long NC, unsigned long long NF, int isEven,
                         unsigned* coarseCells, unsigned* fineCells, unsigned nCells, real omegaC, real omegaF,
                         real* offX, real* offY, real* offZ)
{
    ICellNeigh off { offX, offY, offZ };
    for (unsigned t = 0; t < nCells; ++t) {
        setThread(t);
        scaleFineToCoarseCompressible_Device<false>(distC, distF, nxC, nyC, nzC, nxF, nyF, nzF, NC, NF, isEven != 0,
                                                    coarseCells, fineCells, nCells, omegaC, omegaF, nullptr, nullptr,
                                                    off);
    }
}

// one node of vf::lbm::runK17CompressibleNavierStokes (the shared header)
void REF(vfref_k17_node)(real* f, real omega, real* limiter, real fx, real fy, real fz, real* out4)
{
    vf::lbm::CollisionParameter p;
    for (int d = 0; d < 27; ++d)
        p.distribution[d] = f[d];
    p.omega = omega;
    p.quadricLimiter = limiter;
    p.forceX = fx;
    p.forceY = fy;
    p.forceZ = fz;
    vf::lbm::MacroscopicValues m;
    vf::lbm::TurbulentViscosity tv;
    vf::lbm::runK17CompressibleNavierStokes<vf::lbm::TurbulenceModel::None>(p, m, tv);
    for (int d = 0; d < 27; ++d)
        f[d] = p.distribution[d];
    out4[0] = m.rho;
    out4[1] = m.vx;
    out4[2] = m.vy;
    out4[3] = m.vz;
}

} // extern "C"
