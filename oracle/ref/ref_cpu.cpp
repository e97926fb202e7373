// ref_cpu.cpp -- harness around the reference's CPU K17 path.
//
// TEST INFRASTRUCTURE ONLY (oracle / timed CPU baseline).  Runs the collision
// loop of src/cpu/core/LBM/K17CompressibleNavierStokes.cpp:84-160 on one block
// stored with the reference's own EsoSplit container
// (src/cpu/core/Data/EsoSplit.cpp), calling the reference's shared K17 header.
// The block interior is nx1 x nx2 x nx3 with one ghost layer, as the CPU solver
// allocates it (K17CompressibleNavierStokes.cpp:48-52).  OpenMP splits the
// block along x3; the reference solver runs blocks on OpenMP threads
// (src/cpu/core/Simulation/Simulation.cpp:366-401), so this is the same work
// per thread.  Used to time the reference CPU path on the host.
#include <chrono>
#include <cmath>
#include <memory>

#include <basics/DataTypes.h>
#include <lbm/collision/CollisionParameter.h>
#include <lbm/collision/K17CompressibleNavierStokes.h>
#include <lbm/collision/TurbulentViscosity.h>

#include "Data/EsoSplit.h"
#include "LBM/D3Q27System.h"

#ifdef VF_DOUBLE_ACCURACY
#define REF(name) name##_f64
#else
#define REF(name) name##_f32
#endif

extern "C" {

void* REF(vfref_cpu_block_create)(int nx1, int nx2, int nx3)
{
    auto* e = new EsoSplit((size_t)nx1 + 2, (size_t)nx2 + 2, (size_t)nx3 + 2, (real)0);
    // equilibrium at rest is zero in the shifted variables; add a small
    // deterministic perturbation so the collision works on non-trivial data
    real f[27];
    for (size_t z = 0; z < (size_t)nx3 + 2; ++z)
        for (size_t y = 0; y < (size_t)nx2 + 2; ++y)
            for (size_t x = 0; x < (size_t)nx1 + 2; ++x) {
                for (int d = 0; d < 27; ++d)
                    f[d] = (real)1e-4 * (real)(((x * 7 + y * 13 + z * 29 + (size_t)d * 3) % 17) - 8);
                e->setPreCollisionDistribution(f, x, y, z);
            }
    return e;
}

// A block holding the Taylor-Green vortex of the benchmark workload (n^3
// interior nodes on [-pi, pi)^3, u0, the density of the workload's formula),
// set to the reference CPU path's compressible equilibrium
// (D3Q27System::calcCompFeq) in every node, ghost layer included.  The nodes
// are written in parallel over x3.
void* REF(vfref_cpu_block_create_tgv)(int n, double u0)
{
    const size_t m = (size_t)n + 2;
    auto* e = new EsoSplit(m, m, m, (real)0);
    const double h = 2.0 * M_PI / n;
#pragma omp parallel for schedule(static)
    for (long long z = 0; z < (long long)m; ++z) {
        real f[27];
        for (size_t y = 0; y < m; ++y)
            for (size_t x = 0; x < m; ++x) {
                const double X = -M_PI + h * ((double)x - 1.0), Y = -M_PI + h * ((double)y - 1.0),
                             Z = -M_PI + h * ((double)z - 1.0);
                const real vx = (real)(u0 * std::sin(X) * std::cos(Y) * std::cos(Z));
                const real vy = (real)(-u0 * std::cos(X) * std::sin(Y) * std::cos(Z));
                const real drho = (real)(3.0 * (u0 * u0 / 16.0) * (std::cos(2 * X) + std::cos(2 * Y)) *
                                         (std::cos(2 * Z) + 2.0));
                D3Q27System::calcCompFeq(f, drho, vx, vy, (real)0);
                e->setPreCollisionDistribution(f, x, y, (size_t)z);
            }
    }
    return e;
}

void REF(vfref_cpu_block_free)(void* h) { delete static_cast<EsoSplit*>(h); }

// runs `steps` collision passes over the block interior and returns seconds
double REF(vfref_cpu_block_run)(void* h, int steps, real omega)
{
    EsoSplit* e = static_cast<EsoSplit*>(h);
    const int maxX1 = (int)e->getNX1() - 1, maxX2 = (int)e->getNX2() - 1, maxX3 = (int)e->getNX3() - 1;
    auto t0 = std::chrono::steady_clock::now();
    for (int s = 0; s < steps; ++s) {
#pragma omp parallel for schedule(static)
        for (int x3 = 1; x3 < maxX3; x3++) {
            for (int x2 = 1; x2 < maxX2; x2++) {
                for (int x1 = 1; x1 < maxX1; x1++) {
                    vf::lbm::CollisionParameter parameter;
                    e->getPreCollisionDistribution(parameter.distribution, x1, x2, x3);
                    parameter.forceX = 0;
                    parameter.forceY = 0;
                    parameter.forceZ = 0;
                    parameter.omega = omega;
                    real quadricLimiter[3] = { (real)0.01, (real)0.01, (real)0.01 };
                    parameter.quadricLimiter = quadricLimiter;
                    vf::lbm::MacroscopicValues mv;
                    vf::lbm::TurbulentViscosity tv;
                    vf::lbm::runK17CompressibleNavierStokes<vf::lbm::TurbulenceModel::None>(parameter, mv, tv);
                    e->setPostCollisionDistribution(parameter.distribution, x1, x2, x3);
                }
            }
        }
        e->swap();
    }
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

} // extern "C"
