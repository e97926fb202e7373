// d3q27.cuh -- D3Q27 direction set, lattice weights and esoteric-twist
// addressing shared by every kernel of the library.
//
// Direction numbering, inverse pairs and weights follow
// src/lbm/constants/D3Q27.h:46-106 of VirtualFluids; the array layout
// (f[d * numberOfLBnodes + k], node 0 a dummy) follows
// src/gpu/core/Cuda/CudaMemoryManager.cpp:169 and the twisted views follow
// src/gpu/core/Utilities/KernelUtilities.h:66-125.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace vfb
{
enum Dir : int {
    d000 = 0, dP00, dM00, d0P0, d0M0, d00P, d00M, dPP0, dMM0, dPM0, dMP0, dP0P, dM0M, dP0M, dM0P,
    d0PP, d0MM, d0PM, d0MP, dPPP, dMPP, dPMP, dMMP, dPPM, dMPM, dPMM, dMMM
};

__host__ __device__ constexpr int cx(int d)
{
    constexpr int t[27] = { 0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1 };
    return t[d];
}
__host__ __device__ constexpr int cy(int d)
{
    constexpr int t[27] = { 0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, -1 };
    return t[d];
}
__host__ __device__ constexpr int cz(int d)
{
    constexpr int t[27] = { 0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, 1, 1, 1, -1, -1, -1, -1 };
    return t[d];
}
__host__ __device__ constexpr int inv(int d)
{
    constexpr int t[27] = { 0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17, 26, 25, 24, 23, 22, 21, 20, 19 };
    return t[d];
}
// number of non-zero components (0: rest, 1: face, 2: edge, 3: corner)
__host__ __device__ constexpr int order(int d) { return (cx(d) != 0) + (cy(d) != 0) + (cz(d) != 0); }

// Which of the eight locations of a node direction d is read from before
// collision: bit 0 set for a negative x component (location reached through
// neighborX), bit 1 for y, bit 2 for z.
__host__ __device__ constexpr int loc(int d) { return (cx(d) < 0) | ((cy(d) < 0) << 1) | ((cz(d) < 0) << 2); }

// array slot holding direction d in the even / odd view of the twist
template <bool EVEN>
__host__ __device__ constexpr int slot(int d)
{
    return EVEN ? d : inv(d);
}

template <class R>
__host__ __device__ constexpr R weight(int d)
{
    return order(d) == 0 ? R(8) / R(27) : order(d) == 1 ? R(2) / R(27) : order(d) == 2 ? R(1) / R(54) : R(1) / R(216);
}

// c_d . u summed left to right over the non-zero components (the reference
// writes these as "vx1 - vx2 + vx3" literals, evaluated left to right)
template <class R>
__host__ __device__ __forceinline__ R cdot(int d, R ux, R uy, R uz)
{
    R s = R(0);
    bool first = true;
    if (cx(d) != 0) {
        s = cx(d) > 0 ? ux : -ux;
        first = false;
    }
    if (cy(d) != 0) {
        s = first ? (cy(d) > 0 ? uy : -uy) : (cy(d) > 0 ? s + uy : s - uy);
        first = false;
    }
    if (cz(d) != 0)
        s = first ? (cz(d) > 0 ? uz : -uz) : (cz(d) > 0 ? s + uz : s - uz);
    return s;
}

#ifdef __CUDACC__
// The eight node locations touched by one node (KernelUtilities.h:221-245):
// k[0] the node, k[1] along x, k[2] along y, k[3] along x then y, k[4] along
// z, k[5] along x then z, k[6] along y then z, k[7] along x, y, z.
struct Locs {
    uint32_t k[8];
};

__device__ __forceinline__ Locs listIndices(uint32_t k, const uint32_t* __restrict__ nX,
                                            const uint32_t* __restrict__ nY, const uint32_t* __restrict__ nZ)
{
    Locs L;
    L.k[0] = k;
    L.k[1] = __ldg(nX + k);
    L.k[2] = __ldg(nY + k);
    L.k[4] = __ldg(nZ + k);
    L.k[3] = __ldg(nY + L.k[1]);
    L.k[5] = __ldg(nZ + L.k[1]);
    L.k[6] = __ldg(nZ + L.k[2]);
    L.k[7] = __ldg(nZ + L.k[3]);
    return L;
}
#endif
} // namespace vfb
