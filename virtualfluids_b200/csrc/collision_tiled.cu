// collision_tiled.cu -- the collision plan (tiles of regular nodes, the lane
// list of irregular ones) and the planned entry points; the tile kernels and
// their launchers are in collision_tiled.cuh, instantiated per storage format
// in collision_tiled_<fmt>.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
#include <vector>

#include "collision_tiled.cuh"

namespace vfb
{

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
// direct-load kernel.  Entry 12 (paired, four blocks per SM) is the default
// for FP32, entry 19 (paired, five blocks) for the 16-bit storages and entry 1
// for FP64 (the fastest at Taylor-Green 512^3 on B200: FP16 / FX16 33.5 G node
// updates per second with entry 19 against 32.5 / 31.8 with entry 12);
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
    int def = fp64 ? 1 : storage == VFB_FP32 ? 12 : 19;
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
        e = cudaMalloc(&p.laneLocations, sizeof(uint32_t) * std::max<size_t>(1, 8 * lane.size()));
    if (e == cudaSuccess && !lane.empty())
        if (const int rc = vfb_bc_locations(reinterpret_cast<const int32_t*>(p.laneList), p.nLane, p.nX, p.nY, p.nZ,
                                            p.laneLocations, stream))
            return rc;
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
        const int rc = laneCollision(p.storage, op != Op::K17, &lane, p.laneLocations, stream);
        if (rc != VFB_OK)
            return rc;
    }
    switch (p.storage) {
    case VFB_FP32: return launchTiledFP32(op, p, c, s);
    case VFB_FP64: return launchTiledFP64(op, p, c, s);
    case VFB_FP16: return launchTiledFP16(op, p, c, s);
    case VFB_FX16: return launchTiledFX16(op, p, c, s);
    case VFB_FX16W: return launchTiledFX16W(op, p, c, s);
    default: return launchTiledBF16(op, p, c, s);
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
        cudaFree(p->laneLocations);
        cudaFree(p->error);
        delete p;
        return rc;
    }
    *plan = reinterpret_cast<vfb_collision_plan*>(p);
    return VFB_OK;
}

static void freeEpilogue(vfb_collision_plan_impl& p)
{
    cudaFree(p.epi);
    cudaFree(p.epiNodes);
    cudaFree(p.epiRecords);
    cudaFree(p.epiTileStart);
    cudaFree(p.epiTileNodes);
    p.epi = nullptr;
    p.epiNodes = nullptr;
    p.epiRecords = nullptr;
    p.epiTileStart = nullptr;
    p.epiTileNodes = nullptr;
}

extern "C" int vfb_collision_plan_destroy(vfb_collision_plan* plan)
{
    clearError();
    if (!plan)
        return VFB_OK;
    auto* p = reinterpret_cast<vfb_collision_plan_impl*>(plan);
    cudaFree(p->meta);
    cudaFree(p->laneList);
    cudaFree(p->laneLocations);
    cudaFree(p->error);
    freeEpilogue(*p);
    delete p;
    return VFB_OK;
}

namespace
{
template <class T>
cudaError_t download(std::vector<T>& v, const void* src, size_t n, cudaStream_t s)
{
    v.resize(n);
    return n ? cudaMemcpyAsync(v.data(), src, n * sizeof(T), cudaMemcpyDeviceToHost, s) : cudaSuccess;
}

// the tile configurations whose kernels run the BC epilogue: the paired
// kernels (one stage) and the staged kernels (entries 0-6)
bool epilogueConfig(int c)
{
    return (c >= 0 && c <= 6) || c == 12 || c == 13 || c == 14 || c == 19 || c == 20;
}
} // namespace

extern "C" int vfb_collision_plan_set_bc_epilogue(vfb_collision_plan* plan, const vfb_bc_epilogue_list* lists,
                                                  int nLists, double omega, const int32_t* excludedNodes,
                                                  uint32_t nExcluded, void* stream)
{
    clearError();
    if (!plan)
        return setError(VFB_ERR_INVALID_ARGUMENT, "plan is NULL");
    auto& p = *reinterpret_cast<vfb_collision_plan_impl*>(plan);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (cudaStreamSynchronize(s) != cudaSuccess)
        return setError(VFB_ERR_CUDA, "BC epilogue: %s", cudaGetErrorString(cudaGetLastError()));
    freeEpilogue(p);
    if (nLists == 0)
        return VFB_OK;
    if (nLists < 0 || nLists > kMaxFusedLists || !lists)
        return setError(VFB_ERR_INVALID_ARGUMENT, "the BC epilogue takes 1 to %d lists", kMaxFusedLists);
    if (!epilogueConfig(p.config))
        return setError(VFB_ERR_UNSUPPORTED, "tile configuration %d has no BC epilogue", p.config);
    if (!(omega > 0.0 && omega < 2.0 && omega != 1.0))
        return setError(VFB_ERR_INVALID_ARGUMENT, "omega %g outside (0, 2) or equal to 1", omega);
    if (nExcluded && !excludedNodes)
        return setError(VFB_ERR_INVALID_ARGUMENT, "excludedNodes is NULL");
    for (int l = 0; l < nLists; ++l) {
        const vfb_bc_epilogue_list& L = lists[l];
        if (L.kind < VFB_BC_NOSLIP_INTERPOLATED || L.kind > VFB_BC_VELOCITY_WITH_PRESSURE)
            return setError(VFB_ERR_INVALID_ARGUMENT, "list %d: kind %d is not a post-collision kind", l, L.kind);
        if (L.numberOfBCnodes && (!L.k || !L.q || !L.locations || !L.fused))
            return setError(VFB_ERR_INVALID_ARGUMENT, "list %d: NULL k, q, locations or fused", l);
        const bool velocity = L.kind == VFB_BC_VELOCITY_INTERPOLATED || L.kind == VFB_BC_VELOCITY_BOUNCE_BACK ||
                              L.kind == VFB_BC_VELOCITY_WITH_PRESSURE;
        if (velocity && L.numberOfBCnodes && (!L.Vx || !L.Vy || !L.Vz))
            return setError(VFB_ERR_INVALID_ARGUMENT, "list %d: a velocity kind needs Vx, Vy, Vz", l);
        if (L.numberOfBCnodes > kFusedEntryMask)
            return setError(VFB_ERR_OUT_OF_RANGE, "list %d: too many entries", l);
    }
    const uint64_t N = p.N;
    const bool dbl = p.storage == VFB_FP64;
    std::vector<uint32_t> nx, ny, nz, fl, meta;
    std::vector<int32_t> excl;
    cudaError_t e = download(nx, p.nX, N, s);
    if (e == cudaSuccess) e = download(ny, p.nY, N, s);
    if (e == cudaSuccess) e = download(nz, p.nZ, N, s);
    if (e == cudaSuccess) e = download(fl, p.fluid, p.nFluid, s);
    if (e == cudaSuccess) e = download(meta, p.meta, (size_t)p.nTiles * p.metaWords, s);
    if (e == cudaSuccess) e = download(excl, excludedNodes, nExcluded, s);
    std::vector<std::vector<int32_t>> ks(nLists);
    std::vector<std::vector<uint32_t>> locs(nLists);
    std::vector<std::vector<double>> qs(nLists);
    std::vector<float> qf;
    for (int l = 0; l < nLists && e == cudaSuccess; ++l) {
        const uint32_t n = lists[l].numberOfBCnodes;
        e = download(ks[l], lists[l].k, n, s);
        if (e == cudaSuccess)
            e = download(locs[l], lists[l].locations, 8ull * n, s);
        if (e == cudaSuccess && dbl)
            e = download(qs[l], lists[l].q, 27ull * n, s);
        if (e == cudaSuccess && !dbl) {
            e = download(qf, lists[l].q, 27ull * n, s);
            if (e == cudaSuccess)
                e = cudaStreamSynchronize(s);
            qs[l].assign(qf.begin(), qf.end());
        }
    }
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return setError(VFB_ERR_CUDA, "BC epilogue: copying the lists failed: %s", cudaGetErrorString(e));

    // the bulk tile of every node the tiles collide, and the fluid nodes
    const uint32_t T = p.tileWidth;
    std::vector<int64_t> tileOf(N, -1);
    for (uint32_t t = 0; t < p.nTiles; ++t) {
        const uint32_t* m = meta.data() + (size_t)t * p.metaWords;
        for (uint32_t off = 0; off < T; ++off)
            if ((m[4 + off / 32] >> (off % 32)) & 1u)
                tileOf[(uint64_t)m[0] + off] = t;
    }
    std::vector<uint8_t> isFluid(N, 0), ok(N, 1);
    for (uint32_t k : fl)
        isFluid[k] = 1;
    for (int32_t k : excl)
        if (k >= 0 && (uint64_t)k < N)
            ok[(uint64_t)k] = 0;
    // inverse neighbours: the node whose +axis neighbour is k
    const uint32_t none = 0xffffffffu;
    std::vector<uint32_t> invNb[3] = { std::vector<uint32_t>(N, none), std::vector<uint32_t>(N, none),
                                       std::vector<uint32_t>(N, none) };
    const std::vector<uint32_t>* nb[3] = { &nx, &ny, &nz };
    for (uint64_t k = 0; k < N; ++k)
        for (int ax = 0; ax < 3; ++ax) {
            const uint32_t j = (*nb[ax])[k];
            if (j < N && j != k)
                invNb[ax][j] = (uint32_t)k;
        }
    // a node qualifies when it is a bulk-tile node, not excluded, and every
    // active link of every entry of it writes a cell whose reader (the node C
    // whose location loc(d) is that cell in slot d) is not a fluid node
    for (int l = 0; l < nLists; ++l) {
        const uint32_t n = lists[l].numberOfBCnodes;
        for (uint32_t i = 0; i < n; ++i) {
            const int64_t A = ks[l][i];
            if (A < 0 || (uint64_t)A >= N)
                return setError(VFB_ERR_OUT_OF_RANGE, "list %d entry %u: node %lld outside the lattice", l, i,
                                (long long)A);
            if (tileOf[(uint64_t)A] < 0) {
                ok[(uint64_t)A] = 0;
                continue;
            }
            for (int d = 1; d < 27 && ok[(uint64_t)A]; ++d) {
                const double qd = qs[l][(size_t)d * n + i];
                if (!(qd >= 0.0 && qd <= 1.0))
                    continue;
                uint32_t c = locs[l][(size_t)loc(inv(d)) * n + i]; // the written cell's location index
                const int bits = loc(d);
                for (int ax = 2; ax >= 0 && c != none; --ax)
                    if (bits & (1 << ax))
                        c = invNb[ax][c];
                if (c != none && isFluid[c])
                    ok[(uint64_t)A] = 0;
            }
        }
    }
    // records of the qualifying nodes: per node, in list order, then entry order
    std::vector<std::vector<uint32_t>> byNode; // per qualifying node, in order of first appearance
    std::vector<uint32_t> slotOf(N, none);
    std::vector<uint64_t> nodes;
    for (int l = 0; l < nLists; ++l) {
        const uint32_t n = lists[l].numberOfBCnodes;
        for (uint32_t i = 0; i < n; ++i) {
            const uint64_t A = (uint64_t)ks[l][i];
            if (!ok[A])
                continue;
            if (slotOf[A] == none) {
                slotOf[A] = (uint32_t)byNode.size();
                byNode.emplace_back();
                nodes.push_back(A);
            }
            byNode[slotOf[A]].push_back(((uint32_t)l << 28) | i);
        }
    }
    std::vector<uint32_t> nodeRecord(N, 0u), records;
    std::vector<uint32_t> tileStart(p.nTiles + 1, 0u), tileNodes(nodes.size());
    for (size_t j = 0; j < nodes.size(); ++j) {
        nodeRecord[nodes[j]] = (uint32_t)records.size() + 1u;
        for (size_t r = 0; r < byNode[j].size(); ++r)
            records.push_back(byNode[j][r] | (r + 1 == byNode[j].size() ? kFusedLast : 0u));
        ++tileStart[(size_t)tileOf[nodes[j]] + 1];
    }
    // the BC nodes grouped by tile, in node order within a tile
    for (uint32_t t = 0; t < p.nTiles; ++t)
        tileStart[t + 1] += tileStart[t];
    {
        std::vector<uint64_t> sorted(nodes);
        std::sort(sorted.begin(), sorted.end());
        std::vector<uint32_t> fill(tileStart.begin(), tileStart.end() - 1);
        for (uint64_t A : sorted)
            tileNodes[fill[(size_t)tileOf[A]]++] = (uint32_t)A;
    }
    std::vector<std::vector<uint8_t>> fused(nLists);
    for (int l = 0; l < nLists; ++l) {
        fused[l].resize(lists[l].numberOfBCnodes);
        for (uint32_t i = 0; i < lists[l].numberOfBCnodes; ++i)
            fused[l][i] = ok[(uint64_t)ks[l][i]];
    }
    BcEpilogue h {};
    for (int l = 0; l < nLists; ++l) {
        h.kind[l] = lists[l].kind;
        h.n[l] = lists[l].numberOfBCnodes;
        h.q[l] = lists[l].q;
        h.V[l][0] = lists[l].Vx;
        h.V[l][1] = lists[l].Vy;
        h.V[l][2] = lists[l].Vz;
        h.locations[l] = lists[l].locations;
    }
    h.omega = omega;
    e = upload(&p.epiNodes, nodeRecord, s);
    if (e == cudaSuccess)
        e = upload(&p.epiRecords, records, s);
    if (e == cudaSuccess)
        e = upload(&p.epiTileStart, tileStart, s);
    if (e == cudaSuccess)
        e = upload(&p.epiTileNodes, tileNodes, s);
    h.nodeRecord = p.epiNodes;
    h.records = p.epiRecords;
    if (e == cudaSuccess)
        e = cudaMalloc(&p.epi, sizeof(BcEpilogue));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(p.epi, &h, sizeof(BcEpilogue), cudaMemcpyHostToDevice, s);
    for (int l = 0; l < nLists && e == cudaSuccess; ++l)
        if (lists[l].numberOfBCnodes)
            e = cudaMemcpyAsync(lists[l].fused, fused[l].data(), fused[l].size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        freeEpilogue(p);
        return setError(VFB_ERR_CUDA, "BC epilogue upload failed: %s", cudaGetErrorString(e));
    }
    p.epiCount[0] = nodes.size();
    p.epiCount[1] = records.size();
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

extern "C" int vfb_collision_plan_epilogue_stats(const vfb_collision_plan* plan, unsigned long long* out2)
{
    clearError();
    if (!plan || !out2)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    const auto* p = reinterpret_cast<const vfb_collision_plan_impl*>(plan);
    out2[0] = p->epi ? p->epiCount[0] : 0;
    out2[1] = p->epi ? p->epiCount[1] : 0;
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
