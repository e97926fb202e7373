// sim_state.hpp -- the device-side state of a simulation (per-level arrays,
// BC lists, interface cells) shared by the schedule (simulation.cpp) and the
// adjoint driver (sim_adjoint.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <vector>

#include "../../include/vf_b200.h"

namespace vfb
{
struct AdjointState;
void destroyAdjoint(AdjointState* a);

// a device array owned by the simulation
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    cudaError_t allocate(size_t n)
    {
        bytes = n;
        return cudaMalloc(&ptr, n ? n : 1);
    }
    ~DeviceBuffer()
    {
        if (ptr)
            cudaFree(ptr);
    }
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
};

struct BcListDevice {
    DeviceBuffer k, q, vx, vy, vz;
    DeviceBuffer locations; // 8 * n: the entries' node locations (vfb_bc_locations)
    uint32_t n = 0;
};

// a post-collision list under the plan's BC epilogue: the entries the
// collision kernel does not apply itself, run by the separate BC launch, and
// their indices in the full list (to refresh the velocities)
struct ResidualList {
    BcListDevice list;
    std::vector<uint32_t> index;
};

// interface cells between this level and the next finer one (InterpolationCells
// + ICellNeigh, Calculation.h:72-89)
struct InterfaceDevice {
    DeviceBuffer coarse, fine, offX, offY, offZ, mask;
    DeviceBuffer blocksC, blocksF; // 27 node indices per cell above its coarse / fine base node
    uint32_t n = 0;
};

struct PressureListDevice {
    DeviceBuffer k, kN, rho;
    DeviceBuffer locations; // 16 * n: the eight locations of each node, then of its neighbour
    uint32_t n = 0;
    int direction = 0;
};

// the level's stress list with the wall model's arrays (stressBC and
// wallModel of the reference's level parameters, CudaMemoryManager.cpp:1139-1200)
struct StressListDevice {
    DeviceBuffer k, kN, q, nx, ny, nz, samplingOffset, z0;
    DeviceBuffer el[3], wm[3];    // filter states Vx/Vy/Vz and Vx1/Vy1/Vz1 (zero at start)
    DeviceBuffer uStar, F[3];     // monitors (hasWallModelMonitor)
    DeviceBuffer locations;
    uint32_t n = 0;
};

struct Level {
    unsigned long long N = 0;
    uint32_t nFluid = 0;
    DeviceBuffer dist, nX, nY, nZ, geo, fluid;
    DeviceBuffer nNeg; // the -x-y-z neighbour (non-equilibrium init, enstrophy)
    BcListDevice velocity, noSlip, slip, geometry;
    // the interface lists to the next finer level run in one launch (neither
    // reads what the other writes)
    bool interfaceTogether = false;
    StressListDevice stress;
    // with the plan's BC epilogue: the remaining entries of velocity, no-slip,
    // slip and geometry (in that order), launched after the collision
    bool epilogue = false;
    ResidualList residual[4];
    std::vector<PressureListDevice*> pressure;
    InterfaceDevice coarseToFine, fineToCoarse;
    DeviceBuffer energyNodes; // the kinetic-energy analyzer's node set
    uint32_t nEnergy = 0;
    // drho / vx / vy / vz in the compute precision: the initial fields on their
    // way in and the macroscopic fields on their way out (allocated at first use
    // and kept, so repeated transfers pay no allocation)
    DeviceBuffer fields[4];
    DeviceBuffer outMask; // the output pass's node mask (built at its first call)
    cudaError_t fieldBuffers(size_t bytes)
    {
        for (auto& f : fields)
            if (!f.ptr || f.bytes != bytes) {
                if (f.ptr) {
                    cudaFree(f.ptr);
                    f.ptr = nullptr;
                }
                if (const cudaError_t e = f.allocate(bytes))
                    return e;
            }
        return cudaSuccess;
    }
    double omega = 1.0;
    double forceFactor = 1.0;
    bool isEven = true;
    vfb_collision_plan* plan = nullptr;
    ~Level()
    {
        for (auto* p : pressure)
            delete p;
        if (plan)
            vfb_collision_plan_destroy(plan);
    }
};

// vfb_bc_pressure_noneq reading the list's location table (bc.cu)
int pressureNoneqWithLocations(int storage, const vfb_bc_lattice* lattice, const int32_t* k, const int32_t* kN,
                               const void* rhoBC, uint32_t numberOfBCnodes, int direction, const uint32_t* locations,
                               void* stream);
} // namespace vfb

struct vfb_simulation {
    vfb_sim_params params;
    std::vector<vfb::Level*> levels;
    // captured two-coarse-step graphs, keyed by the parity pattern they start from
    cudaStream_t captureStream = nullptr;
    std::map<unsigned long long, cudaGraphExec_t> graphs;
    unsigned long long stepsRun = 0;
    // level l > 0 runs its two substeps on side[l - 1] beside level l - 1's own
    // step (fork / join events per level; see updateGrid in simulation.cpp)
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> fork, join;
    // the adjoint's checkpoints, tapes and gradients (vfb_sim_adjoint_*)
    vfb::AdjointState* adjoint = nullptr;
    ~vfb_simulation()
    {
        vfb::destroyAdjoint(adjoint);
        for (auto& g : graphs)
            cudaGraphExecDestroy(g.second);
        if (captureStream)
            cudaStreamDestroy(captureStream);
        for (cudaStream_t s : side)
            cudaStreamDestroy(s);
        for (cudaEvent_t e : fork)
            cudaEventDestroy(e);
        for (cudaEvent_t e : join)
            cudaEventDestroy(e);
        for (auto* l : levels)
            delete l;
    }
};
