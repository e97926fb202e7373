// collision_tiled.cuh -- the planned collide + stream path: tile kernels and their
// launchers (the plan and the entry points are in collision_tiled.cu; each
// storage format instantiates the launchers in its own collision_tiled_<fmt>.cu
// so that the formats compile in parallel).
//
// A collision plan (built once per level from the fluid-node list and the
// neighbour arrays) sorts the level's fluid nodes into two kinds of tiles.
// A node is regular when its neighbours follow the lattice strides
// (neighborX = k+1, neighborY = k+sy, neighborZ = k+sz, and likewise for the
// neighbours' neighbours).  Regular nodes are grouped into tiles covering a
// range of T consecutive sparse indices [k0, k0+T) (T = 256, or 128 for FP64);
// for each of the 27 directions the populations of such a range are one
// contiguous run of memory, so the whole tile is fetched with 27 bulk copies
// (cp.async.bulk, about 1 KB each) into shared memory while the block
// collides the previous tile, and no index array is read for it.  A bit mask
// marks which indices of the range are members of the fluid-node list (the
// others -- stoppers, removed or differently tagged nodes -- are skipped).
// Nodes on a periodic wrap stay in the tiles (their wrapped locations are
// read and written in global memory by their own lane).  Irregular nodes
// (next to removed ones, at refinement borders) and sparse ranges go to a
// lane list, collided one node per thread through the index chain by the
// generic kernel.
//
// Two kernels consume the plan.  In the staged kernel (the FP32 / FP64
// default) each block owns shared-memory stages with an mbarrier pair each;
// blocks of a persistent grid stride over the tiles.  In the direct kernel
// (the FP16 / BF16 default, where the collision arithmetic and not the memory
// bounds the step) each block takes one tile and its warps load their values
// from global memory straight into registers.  The arithmetic is the same
// k17Collide / bgkCollide as the generic kernel.  Every population location
// is read and written by exactly one node, and a thread uses only the values
// at its own node's locations, so values a bulk copy fetches for positions no
// thread uses may be stale without harm.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
#include <vector>

#include "bc_entry.cuh"
#include "capi_common.cuh"
#include "collision_math.cuh"
#include "d3q27.cuh"
#include "storage.cuh"
#include "pair32.cuh"
#include "tma.cuh"
#include "pdl.cuh"

namespace vfb
{

// Tile metadata, META_WORDS uint32 per tile (W = warps per tile): word 0 = k0
// (first sparse index of the range), word 1 = bit w set when warp w holds a
// node that wraps around a periodic boundary, words 2..3 unused, words
// 4..4+W = one active-lane mask per warp, then W x-wrap, W y-wrap and W z-wrap
// lane masks.  The producer bulk-copies it into the stage with the tile's
// populations.
//
// A wrap node (the last node of a periodic x line, y column or z pillar) has
// the lattice strides on every axis except the wrapped ones, whose neighbour
// sits a fixed distance back (the wrap offset of that axis).  Its populations
// at the locations on a wrapped axis are not in the tile's bulk copies; its
// lane reads and writes them in global memory directly.

constexpr uint32_t kWaitLimit = 1u << 24; // bounded mbarrier waits

// Tile shape: T nodes (= threads) per tile, STAGES shared-memory stages (a
// prefetch depth of STAGES - 1 tiles), MINB resident blocks the registers are
// sized for.
template <class S, int T_, int STAGES_, int MINB_, int KIND_ = 0>
struct TileCfg {
    static constexpr int KIND = KIND_; // 1: per-warp asynchronous-copy pipeline
    static constexpr int T = T_;
    static constexpr int STAGES = STAGES_;
    static constexpr int MINB = MINB_;
    static constexpr int E = 16 / (int)sizeof(S);                  // elements per 16 bytes
    static constexpr int CAP = ((E - 1 + T + E - 1) / E) * E;      // elements per direction segment
    static constexpr int MASK_WORDS = T / 32;
    static constexpr int META_WORDS = ((4 + 4 * MASK_WORDS + 3) / 4) * 4; // multiple of 4: 16-byte copies
    static constexpr int DATA_BYTES = 27 * CAP * (int)sizeof(S);
    static constexpr int STAGE_BYTES = DATA_BYTES + META_WORDS * 4;
    static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 16 * STAGES; // stages + full / empty mbarriers
    // every bulk copy needs 16-byte aligned addresses and sizes
    static_assert((CAP * (int)sizeof(S)) % 16 == 0, "direction segments must be 16-byte multiples");
    static_assert(DATA_BYTES % 16 == 0, "metadata must start on a 16-byte boundary");
    static_assert((META_WORDS * 4) % 16 == 0, "metadata copy must be a 16-byte multiple");
    static_assert(STAGE_BYTES % 16 == 0, "stages must start on 16-byte boundaries");
    static_assert(T % 32 == 0, "tiles are whole warps");
};

enum class Op { K17, BGK };

template <class S>
struct TiledArgs {
    using R = typename Storage<S>::R;
    S* dist;
    // per direction, for the parity of the launch: the global address of the
    // direction's location of node 0 (dist + slot * N + location stride), the
    // lead of a tile's segment (tiles start at multiples of 16 bytes), the
    // shared-memory offset of node k0 and the bytes of one bulk copy
    S* gbase[27];
    // the last 16-byte aligned start at which a copy of bytes[d] stays inside
    // the population array; a copy that would run past the end starts there
    // instead (the plan guarantees that no lane of such a tile uses it)
    const S* lastSrc[27];
    int lead[27];
    int smemOff[27];
    uint32_t bytes[27];
    uint32_t totalBytes;
    unsigned long long N;
    const uint32_t* __restrict__ meta;
    uint32_t nTiles;
    // per direction: the start of the direction's slot (dist + slot * N); a
    // location's element index within the slot is always in [0, N)
    S* sbase[27];
    // per axis (x, y, z): the location offset of a node, {lattice stride,
    // offset of the periodic image for a node that wraps on that axis}, both
    // modulo 2^32 (node index + offset is the location's index in [0, N))
    uint32_t axisOff[3][2];
    K17Rates<R> rates;
    R fx, fy, fz, gfx, gfy, gfz, forceFactor;
    // the same rates and forces duplicated into register pairs (paired kernel)
    K17Rates<F2> rates2;
    F2 fx2, fy2, fz2;
    R* rho;
    R* vx;
    R* vy;
    R* vz;
    R* bfx;
    R* bfy;
    R* bfz;
    int* errorFlag;
    // the BC epilogue (bc_entry.cuh) or null; the nodes with BC records of
    // tile t are epiTileNodes[epiTileStart[t] .. epiTileStart[t + 1])
    const BcEpilogue* epi;
    const uint32_t* epiTileStart;
    const uint32_t* epiTileNodes;
};

// offset of location loc (bit 0 x, bit 1 y, bit 2 z) from the node for the
// regular lattice strides
__host__ __device__ __forceinline__ uint32_t locShift(int l, uint32_t sy, uint32_t sz)
{
    return (uint32_t)(l & 1) + ((l & 2) ? sy : 0u) + ((l & 4) ? sz : 0u);
}

// location offsets of one lane along x, y and z: the lattice stride, or the
// offset of the periodic image on an axis where the lane's node wraps (wrap
// bits wb: bit 0 x, bit 1 y, bit 2 z)
struct LaneOffsets {
    uint32_t x, y, z;
};

template <class S>
__device__ __forceinline__ LaneOffsets laneOffsets(const TiledArgs<S>& a, int wb)
{
    return { (wb & 1) ? a.axisOff[0][1] : a.axisOff[0][0], (wb & 2) ? a.axisOff[1][1] : a.axisOff[1][0],
             (wb & 4) ? a.axisOff[2][1] : a.axisOff[2][0] };
}

// element index, within its slot, of location l of node k.  The true index is
// in [0, N), so the 32-bit sum with wrap-around is exact.
__device__ __forceinline__ uint32_t locIndex(uint32_t k, LaneOffsets o, int l)
{
    return k + ((l & 1) ? o.x : 0u) + ((l & 2) ? o.y : 0u) + ((l & 4) ? o.z : 0u);
}

// thread 0 arms a stage's "full" barrier and issues the tile's 27 bulk
// copies plus the copy of its metadata
template <class S, class C>
__device__ __forceinline__ void issueTile(const TiledArgs<S>& a, uint32_t tile, uint32_t k0, unsigned char* smem,
                                          int stage, uint64_t* full)
{
    unsigned char* base = smem + stage * C::STAGE_BYTES;
    S* dst = reinterpret_cast<S*>(base);
    tma::mbarArriveExpectTx(&full[stage], a.totalBytes + C::META_WORDS * 4);
    tma::bulkLoad(base + C::DATA_BYTES, a.meta + (size_t)tile * C::META_WORDS, C::META_WORDS * 4, &full[stage]);
#pragma unroll
    for (int d = 0; d < 27; ++d)
    {
        const S* src = a.gbase[d] + (k0 - (uint32_t)a.lead[d]);
        tma::bulkLoad(dst + d * C::CAP, src < a.lastSrc[d] ? src : a.lastSrc[d], a.bytes[d], &full[stage]);
    }
}

template <class S, bool EVEN, Op OP, bool WM, bool BF>
__device__ __forceinline__ void collideNode(const TiledArgs<S>& a, typename Storage<S>::R* f, uint32_t k)
{
    using R = typename Storage<S>::R;
    if (OP == Op::K17) {
        R fx = a.fx, fy = a.fy, fz = a.fz;
        if (BF) {
            fx = (a.gfx + a.bfx[k]) * R(0.5) * a.forceFactor;
            fy = (a.gfy + a.bfy[k]) * R(0.5) * a.forceFactor;
            fz = (a.gfz + a.bfz[k]) * R(0.5) * a.forceFactor;
            a.bfx[k] = R(0);
            a.bfy[k] = R(0);
            a.bfz[k] = R(0);
        }
        R drho, ux, uy, uz;
        k17Collide<R>(f, a.rates, fx, fy, fz, drho, ux, uy, uz);
        if (WM) {
            a.vx[k] = ux;
            a.vy[k] = uy;
            a.vz[k] = uz;
            a.rho[k] = drho;
        }
    } else {
        bgkCollide<R>(f, a.rates.omega);
    }
}

// Pipeline of one block: thread 0 is the producer.  Before refilling a stage
// it waits on the stage's "empty" barrier, on which every warp arrives once it
// has read the stage, then arms the stage's "full" barrier with the tile's
// byte count and issues the 27 bulk copies, STAGES - 1 tiles ahead of the
// consumers.  Every warp waits on "full", moves its 32 nodes' values into
// registers, arrives on "empty", then collides and stores.  Warps never wait
// for each other otherwise.
template <class S, class C, bool EVEN, Op OP, bool WM, bool BF, bool EPI = false>
__global__ void __launch_bounds__(C::T, C::MINB) tiledKernel(const TiledArgs<S> a)
{
    gridDependencyWait();
    using R = typename Storage<S>::R;
    constexpr int WARPS = C::T / 32;
    constexpr int ST = C::STAGES;
    extern __shared__ __align__(128) unsigned char smemRaw[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smemRaw + ST * C::STAGE_BYTES);
    uint64_t* empty = full + ST;
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        for (int i = 0; i < ST; ++i) {
            tma::mbarInit(&full[i], 1);
            tma::mbarInit(&empty[i], WARPS);
        }
        tma::fenceBarrierInit();
    }
    __syncthreads();

    const uint32_t t0 = blockIdx.x, stride = gridDim.x;
    if (t0 >= a.nTiles)
        return;
    const uint32_t mine = (a.nTiles - t0 + stride - 1) / stride; // tiles of this block
    auto k0Of = [&](uint32_t j) { return tma::ldgOrdered(a.meta + (size_t)(t0 + j * stride) * C::META_WORDS); };

    // producer: first STAGES - 1 tiles; pk0 = k0 of the next tile to issue
    uint32_t pk0 = 0;
    if (tid == 0) {
        const uint32_t pre = mine < (uint32_t)(ST - 1) ? mine : (uint32_t)(ST - 1);
        for (uint32_t q = 0; q < pre; ++q)
            issueTile<S, C>(a, t0 + q * stride, k0Of(q), smemRaw, (int)q, full);
        if ((uint32_t)(ST - 1) < mine)
            pk0 = k0Of(ST - 1);
    }
    bool failed = false;

    for (uint32_t j = 0; j < mine; ++j) {
        const int s = (int)(j % ST);
        // producer: tile j + ST - 1 into the stage tile j - 1 used
        if (tid == 0) {
            const uint32_t q = j + ST - 1;
            if (q < mine) {
                const int sq = (int)(q % ST);
                if (q >= (uint32_t)ST && !tma::mbarWait(&empty[sq], ((q - ST) / ST) & 1u, kWaitLimit))
                    failed = true;
                if (!failed) {
                    tma::fenceProxyAsync();
                    issueTile<S, C>(a, t0 + q * stride, pk0, smemRaw, sq, full);
                }
                if (q + 1 < mine)
                    pk0 = k0Of(q + 1);
            }
        }

        const bool ok = tma::mbarWait(&full[s], (j / ST) & 1u, kWaitLimit);
        if (!__all_sync(0xffffffffu, ok) || __any_sync(0xffffffffu, failed)) {
            if (lane == 0)
                atomicExch(a.errorFlag, 1);
            return;
        }
        const unsigned char* stage = smemRaw + s * C::STAGE_BYTES;
        const uint32_t* meta = reinterpret_cast<const uint32_t*>(stage + C::DATA_BYTES);
        const bool active = (meta[4 + warp] >> lane) & 1u;
        const uint32_t k = meta[0] + tid;
        const bool wrapWarp = (meta[1] >> warp) & 1u; // the same for the whole warp
        // wrap bits of this lane: bit 0 x, bit 1 y, bit 2 z
        const int wb = wrapWarp ? (int)((meta[4 + WARPS + warp] >> lane) & 1u) |
                                      (int)(((meta[4 + 2 * WARPS + warp] >> lane) & 1u) << 1) |
                                      (int)(((meta[4 + 3 * WARPS + warp] >> lane) & 1u) << 2)
                                : 0;
        const S* st = reinterpret_cast<const S*>(stage) + tid;
        R f[27];
        if (active) {
            if (!wrapWarp) {
#pragma unroll
                for (int d = 0; d < 27; ++d)
                    f[d] = Storage<S>::load(st + a.smemOff[d], d);
            } else {
                const LaneOffsets o = laneOffsets(a, wb);
#pragma unroll
                for (int d = 0; d < 27; ++d) {
                    const int l = loc(d);
                    f[d] = (l & wb) ? Storage<S>::load(a.sbase[d] + locIndex(k, o, l), d)
                                    : Storage<S>::load(st + a.smemOff[d], d);
                }
            }
        }
        // the stage is free once the warp holds its values: release it before
        // colliding, so the producer refills it while the warp computes (and a
        // wrap lane waiting for its global loads does not hold it)
        __syncwarp();
        if (lane == 0)
            tma::mbarArrive(&empty[s]);
        if (active) {
            collideNode<S, EVEN, OP, WM, BF>(a, f, k);
            if (!wrapWarp) {
#pragma unroll
                for (int d = 0; d < 27; ++d)
                    Storage<S>::store(a.gbase[d] + k, f[inv(d)], d);
            } else {
                const LaneOffsets o = laneOffsets(a, wb);
#pragma unroll
                for (int d = 0; d < 27; ++d)
                    Storage<S>::store(a.sbase[d] + locIndex(k, o, loc(d)), f[inv(d)], d);
            }
            // the node's post-collision BCs, from the values this thread just stored
            if constexpr (EPI) {
                const uint32_t t = t0 + j * stride;
                if (__ldg(a.epiTileStart + t) != __ldg(a.epiTileStart + t + 1))
                    bcEpilogueNode<S, EVEN>(a.dist, a.N, a.epi, k);
            }
        }
    }
}

// Direct form of the planned kernel (a tile configuration with 0 stages): one
// block per tile, every warp loads its nodes' 27 values straight from global
// memory into registers (coalesced: consecutive lanes read consecutive
// addresses of each direction's run), collides and stores.  No producer, no
// shared memory; latency is hidden by the warps resident on the SM.
template <class S, class C, bool EVEN, Op OP, bool WM, bool BF>
__global__ void __launch_bounds__(C::T, C::MINB) directKernel(const TiledArgs<S> a)
{
    gridDependencyWait();
    using R = typename Storage<S>::R;
    constexpr int WARPS = C::T / 32;
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const uint32_t* meta = a.meta + (size_t)blockIdx.x * C::META_WORDS;
    const bool active = (__ldg(meta + 4 + warp) >> lane) & 1u;
    if (!active)
        return;
    const uint32_t k = __ldg(meta) + tid;
    const bool wrapWarp = (__ldg(meta + 1) >> warp) & 1u;
    R f[27];
    if (!wrapWarp) {
#pragma unroll
        for (int d = 0; d < 27; ++d)
            f[d] = Storage<S>::load(a.gbase[d] + k, d);
        collideNode<S, EVEN, OP, WM, BF>(a, f, k);
#pragma unroll
        for (int d = 0; d < 27; ++d)
            Storage<S>::store(a.gbase[d] + k, f[inv(d)], d);
    } else {
        const int wb = (int)((__ldg(meta + 4 + WARPS + warp) >> lane) & 1u) |
                       (int)(((__ldg(meta + 4 + 2 * WARPS + warp) >> lane) & 1u) << 1) |
                       (int)(((__ldg(meta + 4 + 3 * WARPS + warp) >> lane) & 1u) << 2);
        const LaneOffsets o = laneOffsets(a, wb);
#pragma unroll
        for (int d = 0; d < 27; ++d)
            f[d] = Storage<S>::load(a.sbase[d] + locIndex(k, o, loc(d)), d);
        collideNode<S, EVEN, OP, WM, BF>(a, f, k);
#pragma unroll
        for (int d = 0; d < 27; ++d)
            Storage<S>::store(a.sbase[d] + locIndex(k, o, loc(d)), f[inv(d)], d);
    }
}

// Paired direct form (a tile configuration with 1 stage): blocks of T / 2
// threads take one tile each; thread t collides nodes k0 + t and
// k0 + T / 2 + t together in paired FP32 arithmetic (both loads of every
// direction coalesced across the warp).  FP32 arithmetic only (FP32, FP16,
// BF16, FX16 storage); the K17 or the BGK collision.
//
// A warp whose 64 nodes are all active and none wraps (the common case)
// loads and stores without predicates, the second node's address an
// immediate offset from the first's.  Other warps take the general path:
// per-lane predicates and the lanes' location offsets.
template <class S, class C, bool EVEN, Op OP, bool WM, bool BF, bool EPI = false>
__global__ void __launch_bounds__(C::T / 2, C::MINB) pairKernel(const TiledArgs<S> a)
{
    gridDependencyWait();
    constexpr int HALF = C::T / 2;
    constexpr int W2 = HALF / 32; // warps of a block = mask words of one half
    constexpr int WARPS = C::T / 32;
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const uint32_t* meta = a.meta + (size_t)blockIdx.x * C::META_WORDS;
    const uint32_t maskA = __ldg(meta + 4 + warp), maskB = __ldg(meta + 4 + W2 + warp);
    const bool actA = (maskA >> lane) & 1u;
    const bool actB = (maskB >> lane) & 1u;
    // with the BC epilogue every thread reaches the block barrier before it; an
    // inactive lane runs the general path below with all its accesses predicated off
    if (!EPI && !(actA || actB))
        return;
    const uint32_t k0 = __ldg(meta);
    const uint32_t kA = k0 + tid, kB = k0 + HALF + tid;
    const uint32_t wf = __ldg(meta + 1);
    const bool wrap = (((wf >> warp) | (wf >> (W2 + warp))) & 1u) != 0;
    // the same for every lane of the warp
    const bool full = !wrap && (maskA & maskB) == 0xffffffffu;
    LaneOffsets oA = laneOffsets(a, 0), oB = oA;
    if (wrap) {
        auto bitsOf = [&](int word) {
            return (int)((__ldg(meta + 4 + WARPS + word) >> lane) & 1u) |
                   (int)(((__ldg(meta + 4 + 2 * WARPS + word) >> lane) & 1u) << 1) |
                   (int)(((__ldg(meta + 4 + 3 * WARPS + word) >> lane) & 1u) << 2);
        };
        oA = laneOffsets(a, bitsOf(warp));
        oB = laneOffsets(a, bitsOf(W2 + warp));
    }
    // a 16-bit format's storage scale is applied to both nodes in one paired multiply
    using St = Storage<S>;
    F2 f[27];
    if (full) {
#pragma unroll
        for (int d = 0; d < 27; ++d) {
            const S* p = a.gbase[d] + kA;
            f[d] = F2(St::loadRaw(p), St::loadRaw(p + HALF));
        }
    } else {
#pragma unroll
        for (int d = 0; d < 27; ++d) {
            const int l = loc(d);
            const float x = actA ? St::loadRaw(a.sbase[d] + locIndex(kA, oA, l)) : 0.0f;
            const float y = actB ? St::loadRaw(a.sbase[d] + locIndex(kB, oB, l)) : 0.0f;
            f[d] = F2(x, y);
        }
    }
    if (St::scaled) {
#pragma unroll
        for (int d = 0; d < 27; ++d)
            f[d] = f[d] * F2(St::invScale(d));
    }
    F2 fx = a.fx2, fy = a.fy2, fz = a.fz2;
    if (BF) {
        const float h = 0.5f * a.forceFactor;
        fx = F2(actA ? (a.gfx + a.bfx[kA]) * h : 0.0f, actB ? (a.gfx + a.bfx[kB]) * h : 0.0f);
        fy = F2(actA ? (a.gfy + a.bfy[kA]) * h : 0.0f, actB ? (a.gfy + a.bfy[kB]) * h : 0.0f);
        fz = F2(actA ? (a.gfz + a.bfz[kA]) * h : 0.0f, actB ? (a.gfz + a.bfz[kB]) * h : 0.0f);
        if (actA)
            a.bfx[kA] = a.bfy[kA] = a.bfz[kA] = 0.0f;
        if (actB)
            a.bfx[kB] = a.bfy[kB] = a.bfz[kB] = 0.0f;
    }
    F2 drho, ux, uy, uz;
    if constexpr (OP == Op::K17)
        k17Collide<F2>(f, a.rates2, fx, fy, fz, drho, ux, uy, uz);
    else
        bgkCollide<F2>(f, a.rates2.omega);
    if (WM) {
        if (actA) {
            a.rho[kA] = drho.v.x;
            a.vx[kA] = ux.v.x;
            a.vy[kA] = uy.v.x;
            a.vz[kA] = uz.v.x;
        }
        if (actB) {
            a.rho[kB] = drho.v.y;
            a.vx[kB] = ux.v.y;
            a.vy[kB] = uy.v.y;
            a.vz[kB] = uz.v.y;
        }
    }
    if (St::scaled) {
        // f[inv(d)] is stored into the slot of d; both directions have the same weight
#pragma unroll
        for (int d = 0; d < 27; ++d)
            f[d] = f[d] * F2(St::scale(d));
    }
    if (full) {
#pragma unroll
        for (int d = 0; d < 27; ++d) {
            S* p = a.gbase[d] + kA;
            const F2 v = f[inv(d)];
            St::storeRaw(p, v.v.x);
            St::storeRaw(p + HALF, v.v.y);
        }
    } else {
#pragma unroll
        for (int d = 0; d < 27; ++d) {
            const int l = loc(d);
            const F2 v = f[inv(d)];
            if (actA)
                St::storeRaw(a.sbase[d] + locIndex(kA, oA, l), v.v.x);
            if (actB)
                St::storeRaw(a.sbase[d] + locIndex(kB, oB, l), v.v.y);
        }
    }
    // the post-collision BCs of the tile's nodes, shared out over the block
    // once every node of the tile is stored (the barrier makes the block's
    // global stores visible to all its threads).  The values are re-read from
    // L1 / L2, and no lane waits on another lane's BC node of the same warp.
    if constexpr (EPI) {
        const uint32_t b = __ldg(a.epiTileStart + blockIdx.x), e = __ldg(a.epiTileStart + blockIdx.x + 1);
        if (b != e) {
            __syncthreads();
            for (uint32_t j = b + tid; j < e; j += HALF)
                bcEpilogueNode<S, EVEN>(a.dist, a.N, a.epi, __ldg(a.epiTileNodes + j));
        }
    }
}

// Per-thread pipelined form (KIND 1, 4- and 8-byte storage): a persistent
// grid; every thread owns one lane of every tile its block visits and
// prefetches the 27 values of its node of the next tile with cp.async into
// its own shared-memory slots while it collides the current node.  A thread
// reads only what it copied itself, so no barrier of any kind is needed; the
// copies complete through cp.async.wait_group of the same thread.
template <class S, class C, bool EVEN, Op OP, bool WM, bool BF>
__global__ void __launch_bounds__(C::T, C::MINB) asyncKernel(const TiledArgs<S> a)
{
    gridDependencyWait();
    using R = typename Storage<S>::R;
    constexpr int WARPS = C::T / 32;
    extern __shared__ __align__(16) unsigned char smemAsync[];
    S* buf = reinterpret_cast<S*>(smemAsync); // [2][27][T]
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const uint32_t stride = gridDim.x;
    uint32_t tile = blockIdx.x;
    if (tile >= a.nTiles)
        return;
    // head of a tile for this lane: k0, active bit, wrap bits (bit 0 x, 1 y, 2 z)
    auto head = [&](uint32_t t, uint32_t& k0, bool& act, int& wb) {
        const uint32_t* m = a.meta + (size_t)t * C::META_WORDS;
        k0 = __ldg(m);
        act = (__ldg(m + 4 + warp) >> lane) & 1u;
        wb = 0;
        if ((__ldg(m + 1) >> warp) & 1u)
            wb = (int)((__ldg(m + 4 + WARPS + warp) >> lane) & 1u) |
                 (int)(((__ldg(m + 4 + 2 * WARPS + warp) >> lane) & 1u) << 1) |
                 (int)(((__ldg(m + 4 + 3 * WARPS + warp) >> lane) & 1u) << 2);
    };
    // copies of the lane's regular locations only: a wrapped location is read
    // from global memory when the node is collided (its regular address may lie
    // outside the array)
    auto prefetch = [&](int stage, uint32_t k0, bool act, int wb) {
        if (act) {
            S* dst = buf + (size_t)stage * 27 * C::T + tid;
            const uint32_t k = k0 + tid;
#pragma unroll
            for (int d = 0; d < 27; ++d)
                if (!(loc(d) & wb))
                    tma::cpAsync<(int)sizeof(S)>(dst + d * C::T, a.gbase[d] + k);
        }
        tma::cpAsyncCommit();
    };
    uint32_t k0, nk0 = 0;
    bool act, nact = false;
    int wb, nwb = 0;
    head(tile, k0, act, wb);
    prefetch(0, k0, act, wb);
    for (int stage = 0; tile < a.nTiles; tile += stride, stage ^= 1) {
        const uint32_t next = tile + stride;
        if (next < a.nTiles)
            head(next, nk0, nact, nwb);
        else
            nact = false;
        prefetch(stage ^ 1, nk0, nact, nwb); // an empty group at the end keeps the count uniform
        tma::cpAsyncWait<1>();               // this thread's copies of the current tile are done
        if (act) {
            const uint32_t k = k0 + tid;
            const S* src = buf + (size_t)stage * 27 * C::T + tid;
            R f[27];
            const LaneOffsets o = laneOffsets(a, wb);
#pragma unroll
            for (int d = 0; d < 27; ++d) {
                const int l = loc(d);
                if (l & wb)
                    f[d] = Storage<S>::load(a.sbase[d] + locIndex(k, o, l), d);
                else
                    f[d] = Storage<S>::load(src + d * C::T, d);
            }
            collideNode<S, EVEN, OP, WM, BF>(a, f, k);
#pragma unroll
            for (int d = 0; d < 27; ++d)
                Storage<S>::store(a.sbase[d] + locIndex(k, o, loc(d)), f[inv(d)], d);
        }
        k0 = nk0;
        act = nact;
        wb = nwb;
    }
    tma::cpAsyncWait<0>();
}

// ------------------------------------------------------------------ plan --
struct vfb_collision_plan_impl {
    int storage = 0;
    int config = 0;      // index into kTileConfigs
    uint32_t tileWidth = 256;
    uint32_t metaWords = 12;
    unsigned long long N = 0;
    const uint32_t* nX = nullptr;
    const uint32_t* nY = nullptr;
    const uint32_t* nZ = nullptr;
    const uint32_t* fluid = nullptr;
    uint32_t nFluid = 0;
    uint32_t sy = 0, sz = 0;
    long long wrapDelta[3] = { 0, 0, 0 };
    uint32_t* meta = nullptr;
    uint32_t* laneList = nullptr;
    uint32_t* laneLocations = nullptr; // 8 * nLane: the lane list's location table
    uint32_t nTiles = 0;
    uint32_t nLane = 0;
    // tiles, bulk tiles, lane blocks, bulk-fed nodes, wrap nodes served in bulk tiles, nodes collided lane by lane
    unsigned long long stats[6] = { 0, 0, 0, 0, 0, 0 };
    int* error = nullptr;
    // the BC epilogue (vfb_collision_plan_set_bc_epilogue): descriptor, per-node
    // first record, records, per-tile start of the BC nodes and the BC nodes
    // grouped by tile, all device memory
    BcEpilogue* epi = nullptr;
    uint32_t* epiNodes = nullptr;
    uint32_t* epiRecords = nullptr;
    uint32_t* epiTileStart = nullptr;
    uint32_t* epiTileNodes = nullptr;
    unsigned long long epiCount[2] = { 0, 0 }; // nodes, records
};

template <class S, class C, bool EVEN, Op OP, bool WM, bool BF, bool EPI = false>
static int launchTiledT(const TiledArgs<S>& a, cudaStream_t stream)
{
    if constexpr (C::KIND == 1) {
        static int blocks = 0;
        constexpr int smem = 2 * 27 * C::T * (int)sizeof(S);
        if (blocks == 0) {
            cudaError_t e = cudaFuncSetAttribute(asyncKernel<S, C, EVEN, OP, WM, BF>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            if (e != cudaSuccess)
                return setError(VFB_ERR_CUDA, "pipelined kernel shared memory attribute: %s", cudaGetErrorString(e));
            int perSM = 0, device = 0, sms = 0;
            cudaGetDevice(&device);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, asyncKernel<S, C, EVEN, OP, WM, BF>, C::T, smem);
            blocks = std::max(1, perSM) * sms;
        }
        const unsigned grid = (unsigned)std::min<unsigned long long>((unsigned long long)blocks, a.nTiles);
        launchDependent(asyncKernel<S, C, EVEN, OP, WM, BF>, std::max(1u, grid), C::T, smem, stream, a);
        return checkLaunch("pipelined planned collision");
    } else if constexpr (C::STAGES == 1 && sizeof(S) <= 4) {
        launchDependent(pairKernel<S, C, EVEN, OP, WM, BF, EPI>, a.nTiles, C::T / 2, 0, stream, a);
        return checkLaunch("paired planned collision");
    } else if constexpr (C::STAGES == 1) {
        // the paired form computes in FP32: FP64 storage uses the staged kernel
        // of the same tile width (same metadata layout and copy geometry)
        return launchTiledT<S, TileCfg<S, C::T, 2, 3>, EVEN, OP, WM, BF, EPI>(a, stream);
    } else if constexpr (C::STAGES == 0) {
        launchDependent(directKernel<S, C, EVEN, OP, WM, BF>, a.nTiles, C::T, 0, stream, a);
        return checkLaunch("direct planned collision");
    } else {
    static int blocks = 0;
    if (blocks == 0) {
        cudaError_t e = cudaFuncSetAttribute(tiledKernel<S, C, EVEN, OP, WM, BF, EPI>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM_BYTES);
        if (e != cudaSuccess)
            return setError(VFB_ERR_CUDA, "tiled kernel shared memory attribute: %s", cudaGetErrorString(e));
        int perSM = 0, device = 0, sms = 0;
        cudaGetDevice(&device);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, tiledKernel<S, C, EVEN, OP, WM, BF, EPI>, C::T,
                                                      C::SMEM_BYTES);
        blocks = std::max(1, perSM) * sms;
    }
    const unsigned grid = (unsigned)std::min<unsigned long long>((unsigned long long)blocks, a.nTiles);
    launchDependent(tiledKernel<S, C, EVEN, OP, WM, BF, EPI>, std::max(1u, grid), C::T, C::SMEM_BYTES, stream, a);
    return checkLaunch("tiled collision");
    }
}

// the kernels with the BC epilogue, compiled for the default K17 template and
// BGK (the schedule's passes); the epilogue exists for the paired and staged kernels
template <class S, class C>
static int launchEpilogue(Op op, bool even, int tmpl, const TiledArgs<S>& a, cudaStream_t stream)
{
    if constexpr (C::KIND == 1 || C::STAGES == 0) {
        return setError(VFB_ERR_UNSUPPORTED, "this tile configuration has no BC epilogue");
    } else {
        if (op == Op::BGK)
            return even ? launchTiledT<S, C, true, Op::BGK, false, false, true>(a, stream)
                        : launchTiledT<S, C, false, Op::BGK, false, false, true>(a, stream);
        if (tmpl != VFB_TEMPLATE_DEFAULT)
            return setError(VFB_ERR_UNSUPPORTED, "the BC epilogue runs with the default collision template");
        return even ? launchTiledT<S, C, true, Op::K17, false, false, true>(a, stream)
                    : launchTiledT<S, C, false, Op::K17, false, false, true>(a, stream);
    }
}

template <class S, class C>
static int dispatchTiled(Op op, bool even, int tmpl, TiledArgs<S>& a, uint32_t sy, uint32_t sz, uint32_t metaWords,
                  cudaStream_t stream)
{
    if (metaWords != (uint32_t)C::META_WORDS)
        return setError(VFB_ERR_CONFIGURATION, "plan metadata layout does not match the kernel configuration");
    a.totalBytes = 0;
    for (int d = 0; d < 27; ++d) {
        const unsigned long long off = (unsigned long long)(even ? d : inv(d)) * a.N + locShift(loc(d), sy, sz);
        a.gbase[d] = a.dist + off;
        a.sbase[d] = a.dist + (unsigned long long)(even ? d : inv(d)) * a.N;
        a.lead[d] = (int)(off % C::E);
        a.smemOff[d] = d * C::CAP + a.lead[d];
        a.bytes[d] = (uint32_t)(((a.lead[d] + C::T + C::E - 1) / C::E) * C::E * (int)sizeof(S));
        a.lastSrc[d] = a.dist + ((27ull * a.N - a.bytes[d] / sizeof(S)) / C::E) * C::E;
        a.totalBytes += a.bytes[d];
    }
    if (a.epi)
        return launchEpilogue<S, C>(op, even, tmpl, a, stream);
    if (op == Op::BGK)
        return even ? launchTiledT<S, C, true, Op::BGK, false, false>(a, stream)
                    : launchTiledT<S, C, false, Op::BGK, false, false>(a, stream);
    switch (tmpl) {
    case VFB_TEMPLATE_DEFAULT:
        return even ? launchTiledT<S, C, true, Op::K17, false, false>(a, stream)
                    : launchTiledT<S, C, false, Op::K17, false, false>(a, stream);
    case VFB_TEMPLATE_WRITE_MACRO_VARS:
        return even ? launchTiledT<S, C, true, Op::K17, true, false>(a, stream)
                    : launchTiledT<S, C, false, Op::K17, true, false>(a, stream);
    case VFB_TEMPLATE_APPLY_BODY_FORCE:
        return even ? launchTiledT<S, C, true, Op::K17, false, true>(a, stream)
                    : launchTiledT<S, C, false, Op::K17, false, true>(a, stream);
    case VFB_TEMPLATE_ALL_FEATURES:
        return even ? launchTiledT<S, C, true, Op::K17, true, true>(a, stream)
                    : launchTiledT<S, C, false, Op::K17, true, true>(a, stream);
    default: return setError(VFB_ERR_INVALID_ARGUMENT, "invalid collisionTemplate %d", tmpl);
    }
}

// the tuning configurations are compiled for the default K17 and BGK passes
// only; the other templates always use the default shape
template <class S, class C>
static int dispatchTuning(Op op, bool even, int tmpl, TiledArgs<S>& a, uint32_t sy, uint32_t sz, uint32_t metaWords,
                  cudaStream_t stream)
{
    if (metaWords != (uint32_t)C::META_WORDS)
        return setError(VFB_ERR_CONFIGURATION, "plan metadata layout does not match the kernel configuration");
    if (tmpl != VFB_TEMPLATE_DEFAULT && op == Op::K17)
        return setError(VFB_ERR_UNSUPPORTED, "tile configuration supports the default template only");
    a.totalBytes = 0;
    for (int d = 0; d < 27; ++d) {
        const unsigned long long off = (unsigned long long)(even ? d : inv(d)) * a.N + locShift(loc(d), sy, sz);
        a.gbase[d] = a.dist + off;
        a.sbase[d] = a.dist + (unsigned long long)(even ? d : inv(d)) * a.N;
        a.lead[d] = (int)(off % C::E);
        a.smemOff[d] = d * C::CAP + a.lead[d];
        a.bytes[d] = (uint32_t)(((a.lead[d] + C::T + C::E - 1) / C::E) * C::E * (int)sizeof(S));
        a.lastSrc[d] = a.dist + ((27ull * a.N - a.bytes[d] / sizeof(S)) / C::E) * C::E;
        a.totalBytes += a.bytes[d];
    }
    if (a.epi)
        return launchEpilogue<S, C>(op, even, tmpl, a, stream);
    if (op == Op::BGK)
        return even ? launchTiledT<S, C, true, Op::BGK, false, false>(a, stream)
                    : launchTiledT<S, C, false, Op::BGK, false, false>(a, stream);
    return even ? launchTiledT<S, C, true, Op::K17, false, false>(a, stream)
                : launchTiledT<S, C, false, Op::K17, false, false>(a, stream);
}

template <class S>
static int launchTiled(Op op, const vfb_collision_plan_impl& p, const vfb_collision_args* c, cudaStream_t stream)
{
    using R = typename Storage<S>::R;
    TiledArgs<S> a;
    a.dist = static_cast<S*>(c->distributions);
    a.N = p.N;
    a.meta = p.meta;
    a.nTiles = p.nTiles;
    const uint32_t strides[3] = { 1u, p.sy, p.sz };
    for (int ax = 0; ax < 3; ++ax) {
        a.axisOff[ax][0] = strides[ax];
        a.axisOff[ax][1] = (uint32_t)(p.wrapDelta[ax] + (long long)strides[ax]);
    }
    a.rates = makeK17Rates<R>((R)c->omega, (R)c->quadricLimiters[0], (R)c->quadricLimiters[1],
                              (R)c->quadricLimiters[2]);
    a.forceFactor = (R)c->forceFactor;
    a.gfx = (R)c->forces[0];
    a.gfy = (R)c->forces[1];
    a.gfz = (R)c->forces[2];
    a.fx = a.gfx * R(0.5) * a.forceFactor;
    a.fy = a.gfy * R(0.5) * a.forceFactor;
    a.fz = a.gfz * R(0.5) * a.forceFactor;
    if constexpr (sizeof(R) == 4) {
        a.rates2 = pairRates(a.rates);
        a.fx2 = F2(a.fx);
        a.fy2 = F2(a.fy);
        a.fz2 = F2(a.fz);
    }
    a.rho = static_cast<R*>(c->rho);
    a.vx = static_cast<R*>(c->vx);
    a.vy = static_cast<R*>(c->vy);
    a.vz = static_cast<R*>(c->vz);
    a.bfx = static_cast<R*>(c->bodyForceX);
    a.bfy = static_cast<R*>(c->bodyForceY);
    a.bfz = static_cast<R*>(c->bodyForceZ);
    a.errorFlag = p.error;
    a.epi = p.epi;
    a.epiTileStart = p.epiTileStart;
    a.epiTileNodes = p.epiTileNodes;
    if (p.nTiles == 0)
        return VFB_OK;
    const bool even = c->isEvenTimestep != 0;
    const int t = c->collisionTemplate;
    if constexpr (sizeof(S) == 8) {
        switch (p.config) {
        case 6: return dispatchTuning<S, TileCfg<S, 128, 3, 3>>(op, even, t, a, p.sy, p.sz, p.metaWords, stream);
        case 10: return dispatchTuning<S, TileCfg<S, 128, 0, 2>>(op, even, t, a, p.sy, p.sz, p.metaWords, stream);
        case 11: return dispatchTuning<S, TileCfg<S, 128, 0, 3>>(op, even, t, a, p.sy, p.sz, p.metaWords, stream);
        case 17: return dispatchTuning<S, TileCfg<S, 128, 2, 3, 1>>(op, even, t, a, p.sy, p.sz, p.metaWords, stream);
        case 18: return dispatchTuning<S, TileCfg<S, 128, 2, 2, 1>>(op, even, t, a, p.sy, p.sz, p.metaWords, stream);
        default: return dispatchTiled<S, TileCfg<S, 128, 2, 2>>(op, even, t, a, p.sy, p.sz, p.metaWords, stream);
        }
    } else {
        switch (p.config) {
        case 2: return dispatchTuning<S, TileCfg<S, 256, 3, 2>>(op, even, t, a, p.sy, p.sz, p.metaWords, stream);
        case 3: return dispatchTuning<S, TileCfg<S, 192, 3, 3>>(op, even, t, a, p.sy, p.sz, p.metaWords, stream);
        case 4: return dispatchTuning<S, TileCfg<S, 160, 3, 4>>(op, even, t, a, p.sy, p.sz, p.metaWords, stream);
        case 5: return dispatchTuning<S, TileCfg<S, 128, 4, 3>>(op, even, t, a, p.sy, p.sz, p.metaWords, stream);
        case 7: return dispatchTuning<S, TileCfg<S, 128, 0, 4>>(op, even, t, a, p.sy, p.sz, p.metaWords, stream);
        case 12: return dispatchTiled<S, TileCfg<S, 256, 1, 4>>(op, even, t, a, p.sy, p.sz, p.metaWords, stream);
        case 15:
            if constexpr (sizeof(S) == 4)
                return dispatchTuning<S, TileCfg<S, 256, 2, 3, 1>>(op, even, t, a, p.sy, p.sz, p.metaWords, stream);
            else
                return setError(VFB_ERR_UNSUPPORTED, "the pipelined kernel needs 4- or 8-byte storage");
        case 16:
            if constexpr (sizeof(S) == 4)
                return dispatchTuning<S, TileCfg<S, 128, 2, 6, 1>>(op, even, t, a, p.sy, p.sz, p.metaWords, stream);
            else
                return setError(VFB_ERR_UNSUPPORTED, "the pipelined kernel needs 4- or 8-byte storage");
        case 13: return dispatchTiled<S, TileCfg<S, 256, 1, 3>>(op, even, t, a, p.sy, p.sz, p.metaWords, stream);
        case 14: return dispatchTiled<S, TileCfg<S, 256, 1, 2>>(op, even, t, a, p.sy, p.sz, p.metaWords, stream);
        case 19: return dispatchTiled<S, TileCfg<S, 256, 1, 5>>(op, even, t, a, p.sy, p.sz, p.metaWords, stream);
        case 20: return dispatchTiled<S, TileCfg<S, 256, 1, 6>>(op, even, t, a, p.sy, p.sz, p.metaWords, stream);
        case 8: return dispatchTuning<S, TileCfg<S, 256, 0, 3>>(op, even, t, a, p.sy, p.sz, p.metaWords, stream);
        case 9:
            // direct loads, six resident blocks (16-bit storage: all templates)
            if constexpr (sizeof(S) == 2)
                return dispatchTiled<S, TileCfg<S, 128, 0, 6>>(op, even, t, a, p.sy, p.sz, p.metaWords, stream);
            else
                return dispatchTuning<S, TileCfg<S, 128, 0, 6>>(op, even, t, a, p.sy, p.sz, p.metaWords, stream);
        default: return dispatchTiled<S, TileCfg<S, 256, 2, 3>>(op, even, t, a, p.sy, p.sz, p.metaWords, stream);
        }
    }
}


// the launchers of each storage format (collision_tiled_<fmt>.cu)
int launchTiledFP32(Op op, const vfb_collision_plan_impl& p, const vfb_collision_args* c, cudaStream_t s);
int launchTiledFP64(Op op, const vfb_collision_plan_impl& p, const vfb_collision_args* c, cudaStream_t s);
int launchTiledFP16(Op op, const vfb_collision_plan_impl& p, const vfb_collision_args* c, cudaStream_t s);
int launchTiledBF16(Op op, const vfb_collision_plan_impl& p, const vfb_collision_args* c, cudaStream_t s);
int launchTiledFX16(Op op, const vfb_collision_plan_impl& p, const vfb_collision_args* c, cudaStream_t s);
int launchTiledFX16W(Op op, const vfb_collision_plan_impl& p, const vfb_collision_args* c, cudaStream_t s);
// the generic collision over a node list with the list's location table
// (collision.cu; table may be null: the neighbour chain)
int laneCollision(int storage, bool bgk, const vfb_collision_args* args, const uint32_t* table, void* stream);
} // namespace vfb
