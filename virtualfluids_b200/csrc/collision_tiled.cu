// collision_tiled.cu -- the planned collide + stream path.
//
// A collision plan (built once per level from the fluid-node list and the
// neighbour arrays) cuts the fluid-node list into warp tiles of up to 32
// consecutive entries.  A tile whose nodes are consecutive sparse indices
// k0 .. k0+count-1 and whose neighbours follow the lattice strides
// (neighborX = k+1, neighborY = k+sy, neighborZ = k+sz, also for the
// neighbours' neighbours) is "regular": for each of the 27 directions its
// populations form one contiguous run of memory, so the tile is fetched with
// 27 bulk copies (cp.async.bulk) into shared memory one tile ahead of its
// collision, and no index array is read for it.  Lanes whose node breaks the
// strides (a periodic wrap, a node next to a removed node) are exception
// lanes: they follow the neighbour chain and read global memory directly,
// exactly as the generic kernel does.  Tiles whose entries are not
// consecutive, or whose bulk range would leave the array, are processed
// lane by lane like the generic kernel.
//
// Each warp owns two shared-memory stages and an mbarrier per stage; warps of
// a persistent grid stride over the tiles.  The arithmetic is the same
// k17Collide / bgkCollide as the generic kernel, so results are identical.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <vector>

#include "capi_common.cuh"
#include "collision_math.cuh"
#include "d3q27.cuh"
#include "storage.cuh"
#include "tma.cuh"

namespace vfb
{

// tile descriptor: x = first fluid-list entry, y = first node k0,
// z = count | (bulk << 16), w = exception-lane mask
using TileDesc = int4;

constexpr int kTiledWarps = 4;
constexpr int kTiledThreads = 32 * kTiledWarps;
constexpr uint32_t kWaitLimit = 1u << 24; // bounded mbarrier waits

template <class S>
struct Seg {
    static constexpr int E = 16 / (int)sizeof(S);                  // elements per 16 bytes
    static constexpr int CAP = ((E - 1 + 32 + E - 1) / E) * E;     // elements per direction segment
    static constexpr int STAGE_ELEMS = 27 * CAP;
    static constexpr int STAGE_BYTES = STAGE_ELEMS * (int)sizeof(S);
    static constexpr int WARP_BYTES = 2 * STAGE_BYTES + 16;        // two stages + two mbarriers
    static constexpr int BLOCK_BYTES = kTiledWarps * WARP_BYTES;
};

enum class Op { K17, BGK };

template <class S>
struct TiledArgs {
    using R = typename Storage<S>::R;
    S* dist;
    unsigned long long N;
    const uint32_t* __restrict__ nX;
    const uint32_t* __restrict__ nY;
    const uint32_t* __restrict__ nZ;
    const uint32_t* __restrict__ fluid;
    const TileDesc* __restrict__ tiles;
    uint32_t nTiles;
    uint32_t sy, sz;
    K17Rates<R> rates;
    R fx, fy, fz, gfx, gfy, gfz, forceFactor;
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
__device__ __forceinline__ uint32_t locShift(int l, uint32_t sy, uint32_t sz)
{
    return (uint32_t)(l & 1) + ((l & 2) ? sy : 0u) + ((l & 4) ? sz : 0u);
}

template <class S, bool EVEN>
__device__ __forceinline__ void issueTile(const TiledArgs<S>& a, const TileDesc& t, S* stage, uint64_t* bar, int lane)
{
    using G = Seg<S>;
    const uint32_t count = (uint32_t)t.z & 0xffffu;
    uint32_t bytes = 0;
    unsigned long long base = 0;
    uint32_t lead = 0;
    if (lane < 27) {
        base = (unsigned long long)slot<EVEN>(lane) * a.N + (uint32_t)t.y + locShift(loc(lane), a.sy, a.sz);
        lead = (uint32_t)(base % G::E);
        bytes = ((lead + count + G::E - 1) / G::E) * G::E * (uint32_t)sizeof(S);
    }
    const uint32_t total = __reduce_add_sync(0xffffffffu, bytes);
    if (lane == 0)
        tma::mbarArriveExpectTx(bar, total);
    __syncwarp();
    if (lane < 27)
        tma::bulkLoad(stage + lane * G::CAP, a.dist + (base - lead), bytes, bar);
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

template <class S, bool EVEN, Op OP, bool WM, bool BF>
__global__ void __launch_bounds__(kTiledThreads) tiledKernel(const TiledArgs<S> a)
{
    using R = typename Storage<S>::R;
    using G = Seg<S>;
    extern __shared__ __align__(128) unsigned char smemRaw[];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    unsigned char* mine = smemRaw + warp * G::WARP_BYTES;
    S* stages[2] = { reinterpret_cast<S*>(mine), reinterpret_cast<S*>(mine + G::STAGE_BYTES) };
    uint64_t* bars = reinterpret_cast<uint64_t*>(mine + 2 * G::STAGE_BYTES);
    if (lane == 0) {
        tma::mbarInit(&bars[0], 1);
        tma::mbarInit(&bars[1], 1);
        tma::fenceBarrierInit();
    }
    __syncwarp();

    const uint32_t totalWarps = gridDim.x * kTiledWarps;
    uint32_t tIdx = blockIdx.x * kTiledWarps + warp;
    if (tIdx >= a.nTiles)
        return;
    uint32_t uses[2] = { 0, 0 };
    int s = 0;
    TileDesc cur = a.tiles[tIdx];
    if ((cur.z >> 16) & 1)
        issueTile<S, EVEN>(a, cur, stages[s], &bars[s], lane);

    while (true) {
        const uint32_t nIdx = tIdx + totalWarps;
        TileDesc nxt = make_int4(0, 0, 0, 0);
        if (nIdx < a.nTiles) {
            nxt = a.tiles[nIdx];
            if ((nxt.z >> 16) & 1) {
                tma::fenceProxyAsync();
                issueTile<S, EVEN>(a, nxt, stages[s ^ 1], &bars[s ^ 1], lane);
            }
        }

        const uint32_t count = (uint32_t)cur.z & 0xffffu;
        const bool bulk = (cur.z >> 16) & 1;
        const uint32_t exceptions = bulk ? (uint32_t)cur.w : 0xffffffffu;
        if (bulk) {
            const bool ok = __all_sync(0xffffffffu, tma::mbarWait(&bars[s], uses[s] & 1u, kWaitLimit));
            uses[s]++;
            if (!ok) {
                if (lane == 0)
                    atomicExch(a.errorFlag, 1);
                return;
            }
        }
        if ((uint32_t)lane < count) {
            R f[27];
            const bool exc = (exceptions >> lane) & 1u;
            uint32_t k;
            Locs L;
            if (!exc) {
                k = (uint32_t)cur.y + lane;
                const S* st = stages[s];
#pragma unroll
                for (int d = 0; d < 27; ++d) {
                    const unsigned long long base =
                        (unsigned long long)slot<EVEN>(d) * a.N + (uint32_t)cur.y + locShift(loc(d), a.sy, a.sz);
                    f[d] = Storage<S>::load(st + d * G::CAP + (uint32_t)(base % G::E) + lane);
                }
            } else {
                k = __ldg(a.fluid + cur.x + lane);
                L = listIndices(k, a.nX, a.nY, a.nZ);
#pragma unroll
                for (int d = 0; d < 27; ++d)
                    f[d] = Storage<S>::load(a.dist + (unsigned long long)slot<EVEN>(d) * a.N + L.k[loc(d)]);
            }
            collideNode<S, EVEN, OP, WM, BF>(a, f, k);
            if (!exc) {
#pragma unroll
                for (int d = 0; d < 27; ++d)
                    Storage<S>::store(a.dist + (unsigned long long)slot<EVEN>(d) * a.N + k +
                                          locShift(loc(d), a.sy, a.sz),
                                      f[inv(d)]);
            } else {
#pragma unroll
                for (int d = 0; d < 27; ++d)
                    Storage<S>::store(a.dist + (unsigned long long)slot<EVEN>(d) * a.N + L.k[loc(d)], f[inv(d)]);
            }
        }
        __syncwarp();
        if (nIdx >= a.nTiles)
            break;
        tIdx = nIdx;
        cur = nxt;
        s ^= 1;
    }
}


// ------------------------------------------------------------------ plan --
struct vfb_collision_plan_impl {
    int storage = 0;
    unsigned long long N = 0;
    const uint32_t* nX = nullptr;
    const uint32_t* nY = nullptr;
    const uint32_t* nZ = nullptr;
    const uint32_t* fluid = nullptr;
    uint32_t nFluid = 0;
    uint32_t sy = 0, sz = 0;
    TileDesc* tiles = nullptr;
    uint32_t nTiles = 0;
    unsigned long long stats[6] = { 0, 0, 0, 0, 0, 0 }; // tiles, bulk tiles, generic tiles, bulk nodes, exception lanes, generic nodes
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
} // namespace

static int buildPlan(vfb_collision_plan_impl& p, int storage, const vfb_collision_args* a, cudaStream_t stream)
{
    const unsigned long long N = a->numberOfLBnodes;
    const uint32_t nF = a->numberOfFluidNodes;
    std::vector<uint32_t> nx(N), ny(N), nz(N), fl(nF);
    cudaError_t e = cudaMemcpyAsync(nx.data(), a->neighborX, N * 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ny.data(), a->neighborY, N * 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(nz.data(), a->neighborZ, N * 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(fl.data(), a->fluidNodeIndices, (size_t)nF * 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess)
        return setError(VFB_ERR_CUDA, "plan: copying index arrays failed: %s", cudaGetErrorString(e));

    const uint32_t sy = modeStride(fl, ny), sz = modeStride(fl, nz);
    auto regular = [&](uint64_t k) -> bool {
        const uint64_t far = k + 1 + (uint64_t)sy + sz;
        if (far >= N)
            return false;
        return nx[k] == k + 1 && ny[k] == k + sy && nz[k] == k + sz && ny[k + 1] == k + 1 + sy &&
               nz[k + 1] == k + 1 + sz && nz[k + sy] == k + sy + sz && nz[k + 1 + sy] == k + 1 + sy + sz;
    };
    const int esize = vfb_storage_bytes(storage);
    const uint64_t E = 16 / (uint64_t)esize;
    const uint64_t limit = 27ull * N;
    auto bulkInBounds = [&](uint64_t k0, uint32_t count) -> bool {
        for (int even = 0; even < 2; ++even)
            for (int d = 0; d < 27; ++d) {
                const int sl = even ? d : inv(d);
                const int l = loc(d);
                const uint64_t base = (uint64_t)sl * N + k0 + (l & 1) + ((l & 2) ? sy : 0) + ((l & 4) ? sz : 0);
                const uint64_t lead = base % E;
                const uint64_t end = base - lead + ((lead + count + E - 1) / E) * E;
                if (end > limit)
                    return false;
            }
        return true;
    };
    auto runLength = [&](uint32_t i) -> uint32_t {
        uint32_t j = i + 1;
        while (j < nF && j - i < 32 && fl[j] == fl[j - 1] + 1)
            ++j;
        return j - i;
    };

    std::vector<TileDesc> tiles;
    tiles.reserve(nF / 32 + 16);
    uint32_t i = 0;
    while (i < nF) {
        const uint32_t run = runLength(i);
        if (run >= 8) {
            uint32_t mask = 0, regularLanes = 0;
            for (uint32_t t = 0; t < run; ++t) {
                if (regular(fl[i + t]))
                    ++regularLanes;
                else
                    mask |= 1u << t;
            }
            const bool bulk = regularLanes > 0 && bulkInBounds(fl[i], run);
            if (!bulk)
                mask = 0xffffffffu;
            tiles.push_back(make_int4((int)i, (int)fl[i], (int)(run | (bulk ? 1u << 16 : 0u)), (int)mask));
            if (bulk) {
                p.stats[1]++;
                p.stats[3] += regularLanes;
                p.stats[4] += run - regularLanes;
            } else {
                p.stats[2]++;
                p.stats[5] += run;
            }
            i += run;
        } else {
            uint32_t j = i;
            while (j < nF && j - i < 32 && (j == i || runLength(j) < 8))
                ++j;
            tiles.push_back(make_int4((int)i, (int)fl[i], (int)(j - i), (int)0xffffffffu));
            p.stats[2]++;
            p.stats[5] += j - i;
            i = j;
        }
    }
    p.stats[0] = tiles.size();
    p.storage = storage;
    p.N = N;
    p.nX = a->neighborX;
    p.nY = a->neighborY;
    p.nZ = a->neighborZ;
    p.fluid = a->fluidNodeIndices;
    p.nFluid = nF;
    p.sy = sy;
    p.sz = sz;
    p.nTiles = (uint32_t)tiles.size();
    e = cudaMalloc(&p.tiles, sizeof(TileDesc) * std::max<size_t>(1, tiles.size()));
    if (e == cudaSuccess)
        e = cudaMalloc(&p.error, sizeof(int));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(p.tiles, tiles.data(), sizeof(TileDesc) * tiles.size(), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(p.error, 0, sizeof(int), stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess)
        return setError(VFB_ERR_CUDA, "plan: device allocation failed: %s", cudaGetErrorString(e));
    return VFB_OK;
}

template <class S, bool EVEN, Op OP, bool WM, bool BF>
static int launchTiledT(const TiledArgs<S>& a, cudaStream_t stream)
{
    using G = Seg<S>;
    static int blocks = 0;
    if (blocks == 0) {
        cudaError_t e = cudaFuncSetAttribute(tiledKernel<S, EVEN, OP, WM, BF>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, G::BLOCK_BYTES);
        if (e != cudaSuccess)
            return setError(VFB_ERR_CUDA, "tiled kernel shared memory attribute: %s", cudaGetErrorString(e));
        int perSM = 0, device = 0, sms = 0;
        cudaGetDevice(&device);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, tiledKernel<S, EVEN, OP, WM, BF>, kTiledThreads,
                                                      G::BLOCK_BYTES);
        blocks = std::max(1, perSM) * sms;
    }
    const unsigned grid = (unsigned)std::min<unsigned long long>(
        (unsigned long long)blocks, (a.nTiles + kTiledWarps - 1) / (unsigned long long)kTiledWarps);
    tiledKernel<S, EVEN, OP, WM, BF><<<std::max(1u, grid), kTiledThreads, G::BLOCK_BYTES, stream>>>(a);
    return checkLaunch("tiled collision");
}

template <class S>
static int launchTiled(Op op, const vfb_collision_plan_impl& p, const vfb_collision_args* c, cudaStream_t stream)
{
    using R = typename Storage<S>::R;
    TiledArgs<S> a;
    a.dist = static_cast<S*>(c->distributions);
    a.N = p.N;
    a.nX = p.nX;
    a.nY = p.nY;
    a.nZ = p.nZ;
    a.fluid = p.fluid;
    a.tiles = p.tiles;
    a.nTiles = p.nTiles;
    a.sy = p.sy;
    a.sz = p.sz;
    a.rates = makeK17Rates<R>((R)c->omega, (R)c->quadricLimiters[0], (R)c->quadricLimiters[1],
                              (R)c->quadricLimiters[2]);
    a.forceFactor = (R)c->forceFactor;
    a.gfx = (R)c->forces[0];
    a.gfy = (R)c->forces[1];
    a.gfz = (R)c->forces[2];
    a.fx = a.gfx * R(0.5) * a.forceFactor;
    a.fy = a.gfy * R(0.5) * a.forceFactor;
    a.fz = a.gfz * R(0.5) * a.forceFactor;
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
    if (op == Op::BGK)
        return even ? launchTiledT<S, true, Op::BGK, false, false>(a, stream)
                    : launchTiledT<S, false, Op::BGK, false, false>(a, stream);
    switch (c->collisionTemplate) {
    case VFB_TEMPLATE_DEFAULT:
        return even ? launchTiledT<S, true, Op::K17, false, false>(a, stream)
                    : launchTiledT<S, false, Op::K17, false, false>(a, stream);
    case VFB_TEMPLATE_WRITE_MACRO_VARS:
        return even ? launchTiledT<S, true, Op::K17, true, false>(a, stream)
                    : launchTiledT<S, false, Op::K17, true, false>(a, stream);
    case VFB_TEMPLATE_APPLY_BODY_FORCE:
        return even ? launchTiledT<S, true, Op::K17, false, true>(a, stream)
                    : launchTiledT<S, false, Op::K17, false, true>(a, stream);
    case VFB_TEMPLATE_ALL_FEATURES:
        return even ? launchTiledT<S, true, Op::K17, true, true>(a, stream)
                    : launchTiledT<S, false, Op::K17, true, true>(a, stream);
    default: return setError(VFB_ERR_INVALID_ARGUMENT, "invalid collisionTemplate %d", c->collisionTemplate);
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
    switch (p.storage) {
    case VFB_FP32: return launchTiled<float>(op, p, c, s);
    case VFB_FP64: return launchTiled<double>(op, p, c, s);
    case VFB_FP16: return launchTiled<__half>(op, p, c, s);
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
        cudaFree(p->tiles);
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
    cudaFree(p->tiles);
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
