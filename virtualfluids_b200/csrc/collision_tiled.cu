// collision_tiled.cu -- the planned collide + stream path.
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
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
#include <vector>

#include "capi_common.cuh"
#include "collision_math.cuh"
#include "d3q27.cuh"
#include "storage.cuh"
#include "pair32.cuh"
#include "tma.cuh"

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
template <class S, class C, bool EVEN, Op OP, bool WM, bool BF>
__global__ void __launch_bounds__(C::T, C::MINB) tiledKernel(const TiledArgs<S> a)
{
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
// BF16 storage); the K17 collision.
//
// A warp whose 64 nodes are all active and none wraps (the common case)
// loads and stores without predicates, the second node's address an
// immediate offset from the first's.  Other warps take the general path:
// per-lane predicates and the lanes' location offsets.
template <class S, class C, bool EVEN, bool WM, bool BF>
__global__ void __launch_bounds__(C::T / 2, C::MINB) pairKernel(const TiledArgs<S> a)
{
    constexpr int HALF = C::T / 2;
    constexpr int W2 = HALF / 32; // warps of a block = mask words of one half
    constexpr int WARPS = C::T / 32;
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const uint32_t* meta = a.meta + (size_t)blockIdx.x * C::META_WORDS;
    const uint32_t maskA = __ldg(meta + 4 + warp), maskB = __ldg(meta + 4 + W2 + warp);
    const bool actA = (maskA >> lane) & 1u;
    const bool actB = (maskB >> lane) & 1u;
    if (!(actA || actB))
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
    k17Collide<F2>(f, a.rates2, fx, fy, fz, drho, ux, uy, uz);
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
    uint32_t nTiles = 0;
    uint32_t nLane = 0;
    // tiles, bulk tiles, lane blocks, bulk-fed nodes, wrap nodes served in bulk tiles, nodes collided lane by lane
    unsigned long long stats[6] = { 0, 0, 0, 0, 0, 0 };
    int* error = nullptr;
};

namespace
{
// the most frequent value of nb[k] - k over a sample of fluid nodes
uint32_t modeStride(const std::vector<uint32_t>& fluid, const std::vector<uint32_t>& nb)
{
    std::map<long long, size_t> h;
    const size_t step = std::max<size_t>(1, fluid.size() / 4096);
    for (size_t i = 0; i < fluid.size(); i += step) {
        const uint32_t k = fluid[i];
        h[(long long)nb[k] - (long long)k]++;
    }
    long long best = 1;
    size_t n = 0;
    for (auto& kv : h)
        if (kv.second > n && kv.first > 0) {
            n = kv.second;
            best = kv.first;
        }
    return (uint32_t)best;
}

// the most frequent value of nb[k] - k other than the stride over all fluid
// nodes (the wrap offset of a periodic axis), 0 if there is none
long long modeWrap(const std::vector<uint32_t>& fluid, const std::vector<uint32_t>& nb, long long stride)
{
    std::map<long long, size_t> h;
    for (const uint32_t k : fluid) {
        const long long v = (long long)nb[k] - (long long)k;
        if (v != stride)
            h[v]++;
    }
    long long best = 0;
    size_t n = 0;
    for (auto& kv : h)
        if (kv.second > n && kv.first != 0) {
            n = kv.second;
            best = kv.first;
        }
    return best;
}

template <class T>
cudaError_t upload(T** dst, const std::vector<T>& v, cudaStream_t stream)
{
    cudaError_t e = cudaMalloc(dst, sizeof(T) * std::max<size_t>(1, v.size()));
    if (e == cudaSuccess && !v.empty())
        e = cudaMemcpyAsync(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, stream);
    return e;
}
} // namespace

// Tile configurations (tile width, stages, resident blocks) the library is
// compiled for; 0 stages selects the direct-load kernel, 1 stage the paired
// direct-load kernel.  Entry 12 (paired) is the default for FP32, FP16 and
// BF16, entry 1 for FP64 (the fastest at Taylor-Green 512^3 on B200);
// VFB_TILE_CONFIG=<index> selects another one at plan creation (used to tune
// the shape on new hardware).
struct TileConfigInfo {
    int T, stages, minBlocks;
    bool fp64;
};
static const TileConfigInfo kTileConfigs[] = {
    { 256, 2, 3, false }, { 128, 2, 2, true }, { 256, 3, 2, false }, { 192, 3, 3, false },
    { 160, 3, 4, false }, { 128, 4, 3, false }, { 128, 3, 3, true },
    // direct loads (0 stages)
    { 128, 0, 4, false }, { 256, 0, 3, false }, { 128, 0, 6, false }, { 128, 0, 2, true }, { 128, 0, 3, true },
    // paired direct loads (1 stage: T / 2 threads, two nodes each)
    { 256, 1, 4, false }, { 256, 1, 3, false }, { 256, 1, 2, false },
    // per-thread cp.async pipeline (2 shared-memory stages per thread)
    { 256, 2, 3, false }, { 128, 2, 6, false }, { 128, 2, 3, true }, { 128, 2, 2, true },
    // paired, five resident blocks (96 registers, small spills)
    { 256, 1, 5, false },
    // paired, six resident blocks (80 registers)
    { 256, 1, 6, false },
};
static constexpr int kNumTileConfigs = (int)(sizeof(kTileConfigs) / sizeof(kTileConfigs[0]));

static int chooseTileConfig(int storage)
{
    const bool fp64 = storage == VFB_FP64;
    int def = fp64 ? 1 : 12;
    if (const char* env = std::getenv("VFB_TILE_CONFIG")) {
        const int c = std::atoi(env);
        if (c >= 0 && c < kNumTileConfigs && kTileConfigs[c].fp64 == fp64)
            def = c;
    }
    return def;
}

static int buildPlan(vfb_collision_plan_impl& p, int storage, const vfb_collision_args* a, cudaStream_t stream)
{
    p.config = chooseTileConfig(storage);
    p.tileWidth = (uint32_t)kTileConfigs[p.config].T;
    const unsigned long long N = a->numberOfLBnodes;
    const uint32_t nF = a->numberOfFluidNodes;
    std::vector<uint32_t> nx(N), ny(N), nz(N), fl(nF);
    cudaError_t e = cudaMemcpyAsync(nx.data(), a->neighborX, N * 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ny.data(), a->neighborY, N * 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(nz.data(), a->neighborZ, N * 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess && nF)
        e = cudaMemcpyAsync(fl.data(), a->fluidNodeIndices, (size_t)nF * 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess)
        return setError(VFB_ERR_CUDA, "plan: copying index arrays failed: %s", cudaGetErrorString(e));
    for (uint32_t i = 0; i < nF; ++i)
        if (fl[i] >= N)
            return setError(VFB_ERR_OUT_OF_RANGE, "fluid node %u of the list is outside the lattice", fl[i]);

    const int esize = vfb_storage_bytes(storage);
    const uint64_t T = p.tileWidth;
    const uint64_t E = 16 / (uint64_t)esize;
    const uint32_t sy = nF ? modeStride(fl, ny) : 1, sz = nF ? modeStride(fl, nz) : 1;
    // periodic wrap offsets (0: the axis does not wrap)
    const long long wx = modeWrap(fl, nx, 1), wy = modeWrap(fl, ny, sy), wz = modeWrap(fl, nz, sz);
    auto at = [&](const std::vector<uint32_t>& nb, long long k, long long expect) {
        return k >= 0 && k < (long long)N && (long long)nb[k] == expect;
    };
    // wrap bits of node k (bit 0 x, bit 1 y, bit 2 z), or -1 when its
    // neighbours follow neither the strides nor the wrap offsets
    auto classify = [&](uint64_t k) -> int {
        const long long kk = (long long)k;
        int bits = 0;
        long long o[3];
        const std::vector<uint32_t>* nb[3] = { &nx, &ny, &nz };
        const long long stride[3] = { 1, sy, sz }, wrap[3] = { wx, wy, wz };
        for (int ax = 0; ax < 3; ++ax) {
            const long long v = (long long)(*nb[ax])[k] - kk;
            if (v == stride[ax])
                o[ax] = stride[ax];
            else if (wrap[ax] != 0 && v == wrap[ax]) {
                o[ax] = wrap[ax];
                bits |= 1 << ax;
            } else
                return -1;
        }
        const long long k1 = kk + o[0], k2 = kk + o[1], k3 = k1 + o[1];
        if (!at(ny, k1, k3) || !at(nz, k1, k1 + o[2]) || !at(nz, k2, k2 + o[2]) || !at(nz, k3, k3 + o[2]))
            return -1;
        // all eight locations inside the lattice (the wrap lanes address them directly)
        for (int l = 0; l < 8; ++l) {
            const long long kl = kk + ((l & 1) ? o[0] : 0) + ((l & 2) ? o[1] : 0) + ((l & 4) ? o[2] : 0);
            if (kl < 0 || kl >= (long long)N)
                return -1;
        }
        return bits;
    };
    const uint64_t limit = 27ull * N;
    // a copy that would run past the end of the array is moved back inside it
    // by the kernel, so the tile may only hold lanes that do not read it (lanes
    // that wrap on an axis of the copy's location)
    auto bulkUsable = [&](uint64_t k0, const uint64_t* first, const uint64_t* last) -> bool {
        if (N * 27ull < T + 2 * E)
            return false;
        for (int even = 0; even < 2; ++even)
            for (int d = 0; d < 27; ++d) {
                const uint64_t base = (uint64_t)(even ? d : inv(d)) * N + k0 + locShift(loc(d), sy, sz);
                const uint64_t lead = base % E;
                if (base - lead + ((lead + T + E - 1) / E) * E <= limit)
                    continue;
                for (const uint64_t* q = first; q != last; ++q)
                    if ((loc(d) & (int)(*q & 7u)) == 0)
                        return false;
            }
        return true;
    };

    // classified list members as (k << 3 | wrap bits), ascending; the others go lane by lane
    std::vector<uint64_t> cand;
    std::vector<uint32_t> lane;
    cand.reserve(nF);
    for (uint32_t i = 0; i < nF; ++i) {
        const int bits = classify(fl[i]);
        if (bits >= 0)
            cand.push_back(((uint64_t)fl[i] << 3) | (uint64_t)bits);
        else
            lane.push_back(fl[i]);
    }
    std::sort(cand.begin(), cand.end());
    for (size_t i = 1; i < cand.size(); ++i)
        if ((cand[i] >> 3) == (cand[i - 1] >> 3))
            return setError(VFB_ERR_INVALID_ARGUMENT, "the fluid-node list holds a node twice");

    std::vector<uint32_t> meta;
    const uint64_t words = T / 32;
    const uint64_t metaWords = ((4 + 4 * words + 3) / 4) * 4; // TileCfg::META_WORDS
    const uint64_t minActive = T / 4;
    size_t i = 0;
    while (i < cand.size()) {
        const uint64_t first = cand[i] >> 3;
        const uint64_t k0 = first - first % E; // bulk sources then share one lead per direction
        size_t j = i;
        while (j < cand.size() && (cand[j] >> 3) < k0 + T)
            ++j;
        const uint64_t active = j - i;
        if (active >= minActive && bulkUsable(k0, cand.data() + i, cand.data() + j)) {
            const size_t base = meta.size();
            meta.resize(base + metaWords, 0u);
            meta[base] = (uint32_t)k0;
            for (size_t q = i; q < j; ++q) {
                const uint64_t off = (cand[q] >> 3) - k0;
                const uint32_t bits = (uint32_t)(cand[q] & 7u), w = (uint32_t)(off / 32), b = 1u << (off % 32);
                meta[base + 4 + w] |= b;
                for (int ax = 0; ax < 3; ++ax)
                    if (bits & (1u << ax))
                        meta[base + 4 + (1 + ax) * words + w] |= b;
                if (bits) {
                    meta[base + 1] |= 1u << w;
                    p.stats[4]++;
                }
            }
            p.stats[1]++;
            p.stats[3] += active;
        } else {
            for (size_t q = i; q < j; ++q)
                lane.push_back((uint32_t)(cand[q] >> 3));
        }
        i = j;
    }
    // the nodes left over are collided one per thread by the generic kernel
    std::sort(lane.begin(), lane.end());
    p.stats[2] = (lane.size() + T - 1) / T;
    p.stats[5] = lane.size();
    p.stats[0] = p.stats[1];

    p.storage = storage;
    p.N = N;
    p.nX = a->neighborX;
    p.nY = a->neighborY;
    p.nZ = a->neighborZ;
    p.fluid = a->fluidNodeIndices;
    p.nFluid = nF;
    p.sy = sy;
    p.sz = sz;
    p.wrapDelta[0] = wx ? wx - 1 : 0;
    p.wrapDelta[1] = wy ? wy - (long long)sy : 0;
    p.wrapDelta[2] = wz ? wz - (long long)sz : 0;
    p.nTiles = (uint32_t)p.stats[1];
    p.metaWords = (uint32_t)metaWords;
    p.nLane = (uint32_t)lane.size();
    e = upload(&p.meta, meta, stream);
    if (e == cudaSuccess)
        e = upload(&p.laneList, lane, stream);
    if (e == cudaSuccess)
        e = cudaMalloc(&p.error, sizeof(int));
    if (e == cudaSuccess)
        e = cudaMemsetAsync(p.error, 0, sizeof(int), stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess)
        return setError(VFB_ERR_CUDA, "plan: device allocation failed: %s", cudaGetErrorString(e));
    return VFB_OK;
}

template <class S, class C, bool EVEN, Op OP, bool WM, bool BF>
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
        asyncKernel<S, C, EVEN, OP, WM, BF><<<std::max(1u, grid), C::T, smem, stream>>>(a);
        return checkLaunch("pipelined planned collision");
    } else if constexpr (C::STAGES == 1 && OP == Op::K17 && sizeof(S) <= 4) {
        pairKernel<S, C, EVEN, WM, BF><<<a.nTiles, C::T / 2, 0, stream>>>(a);
        return checkLaunch("paired planned collision");
    } else if constexpr (C::STAGES == 1) {
        // the paired form is K17 only: other operators use the staged kernel of
        // the same tile width (same metadata layout and copy geometry)
        return launchTiledT<S, TileCfg<S, C::T, 2, 3>, EVEN, OP, WM, BF>(a, stream);
    } else if constexpr (C::STAGES == 0) {
        directKernel<S, C, EVEN, OP, WM, BF><<<a.nTiles, C::T, 0, stream>>>(a);
        return checkLaunch("direct planned collision");
    } else {
    static int blocks = 0;
    if (blocks == 0) {
        cudaError_t e = cudaFuncSetAttribute(tiledKernel<S, C, EVEN, OP, WM, BF>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM_BYTES);
        if (e != cudaSuccess)
            return setError(VFB_ERR_CUDA, "tiled kernel shared memory attribute: %s", cudaGetErrorString(e));
        int perSM = 0, device = 0, sms = 0;
        cudaGetDevice(&device);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, tiledKernel<S, C, EVEN, OP, WM, BF>, C::T,
                                                      C::SMEM_BYTES);
        blocks = std::max(1, perSM) * sms;
    }
    const unsigned grid = (unsigned)std::min<unsigned long long>((unsigned long long)blocks, a.nTiles);
    tiledKernel<S, C, EVEN, OP, WM, BF><<<std::max(1u, grid), C::T, C::SMEM_BYTES, stream>>>(a);
    return checkLaunch("tiled collision");
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

static int runPlanned(Op op, const vfb_collision_plan* plan, const vfb_collision_args* c, void* stream)
{
    clearError();
    if (!plan || !c)
        return setError(VFB_ERR_INVALID_ARGUMENT, "plan or args is NULL");
    const auto& p = *reinterpret_cast<const vfb_collision_plan_impl*>(plan);
    if (c->numberOfLBnodes != p.N || c->neighborX != p.nX || c->neighborY != p.nY || c->neighborZ != p.nZ ||
        c->fluidNodeIndices != p.fluid || c->numberOfFluidNodes != p.nFluid)
        return setError(VFB_ERR_INVALID_ARGUMENT, "args do not match the index arrays the plan was built for");
    if (!c->distributions || (reinterpret_cast<uintptr_t>(c->distributions) & 15u) != 0)
        return setError(VFB_ERR_INVALID_ARGUMENT, "distributions must be 16-byte aligned");
    if (!(c->omega > 0.0 && c->omega < 2.0))
        return setError(VFB_ERR_INVALID_ARGUMENT, "omega %g outside (0, 2)", c->omega);
    if (op == Op::K17) {
        const int t = c->collisionTemplate;
        if ((t == VFB_TEMPLATE_WRITE_MACRO_VARS || t == VFB_TEMPLATE_ALL_FEATURES) &&
            (!c->rho || !c->vx || !c->vy || !c->vz))
            return setError(VFB_ERR_INVALID_ARGUMENT, "template %d needs rho/vx/vy/vz", t);
        if ((t == VFB_TEMPLATE_APPLY_BODY_FORCE || t == VFB_TEMPLATE_ALL_FEATURES) &&
            (!c->bodyForceX || !c->bodyForceY || !c->bodyForceZ))
            return setError(VFB_ERR_INVALID_ARGUMENT, "template %d needs bodyForceX/Y/Z", t);
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (p.nLane) {
        // the irregular nodes, one per thread through the index chain
        vfb_collision_args lane = *c;
        lane.fluidNodeIndices = p.laneList;
        lane.numberOfFluidNodes = p.nLane;
        const int rc = op == Op::K17 ? vfb_k17_collision(p.storage, &lane, stream) : vfb_bgk_collision(p.storage, &lane, stream);
        if (rc != VFB_OK)
            return rc;
    }
    switch (p.storage) {
    case VFB_FP32: return launchTiled<float>(op, p, c, s);
    case VFB_FP64: return launchTiled<double>(op, p, c, s);
    case VFB_FP16: return launchTiled<__half>(op, p, c, s);
    case VFB_FX16: return launchTiled<int16_t>(op, p, c, s);
    default: return launchTiled<__nv_bfloat16>(op, p, c, s);
    }
}

} // namespace vfb

using namespace vfb;

extern "C" int vfb_collision_plan_create(int storage, const vfb_collision_args* args, vfb_collision_plan** plan,
                                         void* stream)
{
    clearError();
    if (!args || !plan)
        return setError(VFB_ERR_INVALID_ARGUMENT, "args or plan is NULL");
    *plan = nullptr;
    if (vfb_storage_bytes(storage) == 0)
        return setError(VFB_ERR_INVALID_ARGUMENT, "unknown storage %d", storage);
    if (!args->neighborX || !args->neighborY || !args->neighborZ || (!args->fluidNodeIndices && args->numberOfFluidNodes))
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL neighbor or fluid-node array");
    if (args->numberOfLBnodes < 2 || args->numberOfLBnodes > 0xffffffffull)
        return setError(VFB_ERR_OUT_OF_RANGE, "numberOfLBnodes %llu outside [2, 2^32)", args->numberOfLBnodes);
    auto* p = new vfb_collision_plan_impl;
    const int rc = buildPlan(*p, storage, args, static_cast<cudaStream_t>(stream));
    if (rc != VFB_OK) {
        cudaFree(p->meta);
        cudaFree(p->laneList);
        cudaFree(p->error);
        delete p;
        return rc;
    }
    *plan = reinterpret_cast<vfb_collision_plan*>(p);
    return VFB_OK;
}

extern "C" int vfb_collision_plan_destroy(vfb_collision_plan* plan)
{
    clearError();
    if (!plan)
        return VFB_OK;
    auto* p = reinterpret_cast<vfb_collision_plan_impl*>(plan);
    cudaFree(p->meta);
    cudaFree(p->laneList);
    cudaFree(p->error);
    delete p;
    return VFB_OK;
}

extern "C" int vfb_collision_plan_stats(const vfb_collision_plan* plan, unsigned long long* out6)
{
    clearError();
    if (!plan || !out6)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    const auto* p = reinterpret_cast<const vfb_collision_plan_impl*>(plan);
    for (int i = 0; i < 6; ++i)
        out6[i] = p->stats[i];
    return VFB_OK;
}

extern "C" int vfb_collision_plan_check(const vfb_collision_plan* plan, void* stream)
{
    clearError();
    if (!plan)
        return setError(VFB_ERR_INVALID_ARGUMENT, "plan is NULL");
    const auto* p = reinterpret_cast<const vfb_collision_plan_impl*>(plan);
    int flag = 0;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemcpyAsync(&flag, p->error, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return setError(VFB_ERR_CUDA, "plan check: %s", cudaGetErrorString(e));
    if (flag)
        return setError(VFB_ERR_CUDA, "a bounded wait for a bulk copy ran out in the tiled collision kernel");
    return VFB_OK;
}

extern "C" int vfb_k17_collision_planned(const vfb_collision_plan* plan, const vfb_collision_args* args, void* stream)
{
    return runPlanned(Op::K17, plan, args, stream);
}

extern "C" int vfb_bgk_collision_planned(const vfb_collision_plan* plan, const vfb_collision_args* args, void* stream)
{
    return runPlanned(Op::BGK, plan, args, stream);
}
