// adjoint.cuh -- kernels of the adjoint (reverse-mode) time step, launched by
// the simulation's adjoint driver (sim_adjoint.cu, vfb_sim_adjoint_*).
//
// The forward step they differentiate is the single-level UpdateGrid27 step
// (UpdateGrid27.cpp:54-96): K17 collision over the fluid list with in-place
// esoteric-twist streaming (K17CompressibleNavierStokes.h:87-591 through
// RunCollision.cuh:74-143), the post-collision lists (velocity, no-slip,
// geometry: VelocityInterpolatedCompressible.cu:44-418,
// NoSlipInterpolatedCompressible.cu:44-378), the parity swap and the
// non-equilibrium pressure list (PressureNonEquilibriumCompressible.cu:45-311).
// The reference has no adjoint; these are the transposed Jacobians of those
// maps.
//
// Every forward kernel here is the library's forward arithmetic (the same
// operator templates and BC formulas) plus an optional record of its inputs:
// the collision writes the 27 pre-collision values of each fluid node to a
// tape (tape[d * n + i] for fluid-list entry i), a BC kernel the 27 values it
// reads per BC node (rec[d * n + i]).  The adjoint kernels read those records
// and the adjoint array lam (the layout of the populations).
//
// Overwritten cells: a BC writes some cells without reading them, so its
// adjoint runs in two launches: "gather" moves lam at every written cell into
// tmp[d * n + i] and clears the cell; "scatter" adds the contributions of the
// node's formula to the cells it read.  The entries of a list write disjoint
// cells, so the gather does not race; the scatters add with atomics, since a
// node may appear in a list more than once (edge nodes of two walls, each
// entry with the directions of its wall) and two pressure nodes may share a
// neighbour.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "bc_math.cuh"
#include "collision_math.cuh"

namespace vfb
{
namespace adjoint
{
// blocks of the collision adjoint (its block partial sums of the force adjoint)
unsigned collisionBlocks(uint32_t nFluid);

// forward K17 collision over the fluid list; tape may be null; loc is the
// fluid list's location table (8 * nFluid, vfb_bc_locations layout) or null
template <class R>
int collision(R* dist, unsigned long long N, const uint32_t* nX, const uint32_t* nY, const uint32_t* nZ,
              const uint32_t* fluid, const uint32_t* loc, uint32_t nFluid, const K17Rates<R>& rates, R fx, R fy, R fz,
              bool even, R* tape, cudaStream_t s);

// adjoint of the collision: lam in place; partials[3 * b + c] accumulate the
// block sums of the adjoint of the half force (fx, fy, fz) (the caller
// clears them before the first step and reduces them after the last)
template <class R>
int collisionAdjoint(R* lam, unsigned long long N, const uint32_t* nX, const uint32_t* nY, const uint32_t* nZ,
                     const uint32_t* fluid, const uint32_t* loc, uint32_t nFluid, const K17Rates<R>& rates, R fx,
                     R fy, R fz, bool even, const R* tape, double* partials, cudaStream_t s);

// forward post-collision BC (kind VFB_BC_VELOCITY_INTERPOLATED or
// VFB_BC_NOSLIP_INTERPOLATED); rec may be null; table is the list's location
// table (vfb_bc_locations) or null
template <class R>
int postBC(int kind, R* dist, const BcLattice<R>& lat, const int32_t* k, const uint32_t* table, const R* q, uint32_t n,
           const R* Vx, const R* Vy, const R* Vz, bool even, R* rec, cudaStream_t s);

// adjoint of postBC: gather then scatter; gV (3 n doubles: x block, y block,
// z block) accumulates the adjoint of the BC velocities (velocity kind)
template <class R>
int postBCAdjoint(int kind, R* lam, const BcLattice<R>& lat, const int32_t* k, const uint32_t* table, const R* q,
                  uint32_t n, const R* Vx, const R* Vy, const R* Vz, bool even, const R* rec, R* tmp, double* gV,
                  cudaStream_t s);

// Several post-collision lists of one step in one launch (the caller has
// checked that no list writes a cell another list reads or writes).  rec is
// the list's record slot of the step (forward: written, may be null;
// adjoint: read), tmp and gV as for postBCAdjoint.
constexpr int kMaxPostLists = 3;
template <class R>
struct PostList {
    int kind;
    const int32_t* k;
    const uint32_t* table;
    const R* q;
    uint32_t n;
    const R* Vx;
    const R* Vy;
    const R* Vz;
    R* rec;
    R* tmp;
    double* gV;
};
template <class R>
struct PostLists {
    int count = 0;
    unsigned firstBlock[kMaxPostLists] = { 0, 0, 0 }; // filled by the launchers
    PostList<R> list[kMaxPostLists];
};
template <class R>
int postBCLists(R* dist, const BcLattice<R>& lat, PostLists<R> lists, bool even, cudaStream_t s);
template <class R>
int postBCAdjointLists(R* lam, const BcLattice<R>& lat, PostLists<R> lists, bool even, cudaStream_t s);
// forward non-equilibrium pressure BC (after the swap); rec may be null
template <class R>
int pressureBC(R* dist, const BcLattice<R>& lat, const int32_t* k, const int32_t* kN, const R* rhoBC, uint32_t n,
               int direction, bool even, R* rec, cudaStream_t s);

template <class R>
int pressureBCAdjoint(R* lam, const BcLattice<R>& lat, const int32_t* k, const int32_t* kN, const R* rhoBC,
                      uint32_t n, int direction, bool even, const R* rec, R* tmp, cudaStream_t s);

// objective J = sum_j wx_j ux + wy_j uy + wz_j uz over nodes[j], u = j / (1 +
// drho) of the populations of parity `even`: block partials of J into
// partials[b]; with lam non-null, seed * dJ/df is added to lam as well
template <class R>
int objective(const R* dist, unsigned long long N, const uint32_t* nX, const uint32_t* nY, const uint32_t* nZ,
              const uint32_t* nodes, const double* wx, const double* wy, const double* wz, uint32_t n, bool even,
              double* partials, R* lam, double seed, cudaStream_t s);
unsigned objectiveBlocks(uint32_t n);

// acc[c] += scale * sum over b of partials[width * b + c], c < width, in block order
int reducePartials(const double* partials, unsigned blocks, int width, double* acc, double scale, cudaStream_t s);
} // namespace adjoint
} // namespace vfb
