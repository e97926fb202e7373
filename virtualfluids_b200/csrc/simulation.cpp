// simulation.cpp -- the host side of the time step: level data, kernel
// selection and the recursive per-level substep schedule of the reference's
// UpdateGrid27 (src/gpu/core/Calculation/UpdateGrid27.cpp:54-96,228-308),
// calling the kernels through the library's own C ABI.
//
// Everything here is stream ordered on the caller's stream; the host never
// waits except where a call returns data to the host.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "capi_common.cuh"
#include "sim_state.hpp"

namespace vfb
{
namespace
{

int elementBytes(int storage) { return vfb_storage_bytes(storage); }
bool computeIsDouble(int storage) { return storage == VFB_FP64; }

} // namespace
} // namespace vfb


namespace vfb
{
namespace
{

// copies a grid array of `name` (count elements of elemSize bytes) to the host
bool gridArray(void* grid, int level, const char* name, std::vector<char>& out, long long& count, int& elemSize)
{
    count = vfb_grid_count(grid, level, name);
    elemSize = vfb_grid_elem_size(grid, level, name);
    if (count < 0 || elemSize <= 0)
        return false;
    out.resize((size_t)count * elemSize);
    return vfb_grid_copy(grid, level, name, out.empty() ? nullptr : out.data()) == VFB_OK;
}

cudaError_t uploadRaw(DeviceBuffer& b, const void* host, size_t bytes, cudaStream_t s)
{
    cudaError_t e = b.allocate(bytes);
    if (e == cudaSuccess && bytes)
        e = cudaMemcpyAsync(b.ptr, host, bytes, cudaMemcpyHostToDevice, s);
    return e;
}

// uploads a double array as the compute precision of the storage
// Host doubles into a device array of the compute precision.  A divisor other
// than 1 divides every value after the conversion, in the compute precision, as
// the reference scales the geometry velocities (GridGenerator.cpp:507-513).
cudaError_t uploadReal(DeviceBuffer& b, const std::vector<char>& raw, int storage, cudaStream_t s,
                       std::vector<std::vector<char>>& keep, double divisor = 1.0)
{
    const size_t n = raw.size() / sizeof(double);
    const double* src = reinterpret_cast<const double*>(raw.data());
    keep.emplace_back();
    std::vector<char>& host = keep.back();
    if (computeIsDouble(storage)) {
        host = raw;
        if (divisor != 1.0) {
            double* dst = reinterpret_cast<double*>(host.data());
            for (size_t i = 0; i < n; ++i)
                dst[i] = dst[i] / divisor;
        }
    } else {
        host.resize(n * sizeof(float));
        float* dst = reinterpret_cast<float*>(host.data());
        const float d = (float)divisor;
        for (size_t i = 0; i < n; ++i)
            dst[i] = divisor != 1.0 ? (float)src[i] / d : (float)src[i];
    }
    return uploadRaw(b, host.data(), host.size(), s);
}

int uploadLevel(Level& L, void* grid, int level, int storage, double geometryVelocityDivisor, cudaStream_t s,
                std::vector<std::vector<char>>& keep)
{
    std::vector<char> raw;
    long long count = 0;
    int es = 0;
    auto fail = [&](const char* what) { return setError(VFB_ERR_CONFIGURATION, "grid level %d: array %s", level, what); };
    auto need = [&](const char* name, int elem) -> bool {
        return gridArray(grid, level, name, raw, count, es) && es == elem;
    };
    cudaError_t e = cudaSuccess;
    if (!need("geo", 4))
        return fail("geo");
    L.N = (unsigned long long)count;
    keep.push_back(raw);
    e = uploadRaw(L.geo, keep.back().data(), raw.size(), s);
    const char* nb[3] = { "neighborX", "neighborY", "neighborZ" };
    DeviceBuffer* nbuf[3] = { &L.nX, &L.nY, &L.nZ };
    for (int i = 0; i < 3 && e == cudaSuccess; ++i) {
        if (!need(nb[i], 4) || (unsigned long long)count != L.N)
            return fail(nb[i]);
        keep.push_back(raw);
        e = uploadRaw(*nbuf[i], keep.back().data(), raw.size(), s);
    }
    if (e == cudaSuccess) {
        if (!need("fluid", 4))
            return fail("fluid");
        L.nFluid = (uint32_t)count;
        keep.push_back(raw);
        e = uploadRaw(L.fluid, keep.back().data(), raw.size(), s);
    }
    // compacted BC lists: k (int32), q (27 * n doubles), velocities
    auto list = [&](const std::string& prefix, BcListDevice& B, bool velocity, double divisor = 1.0) -> int {
        if (!need((prefix + ".k").c_str(), 4))
            return fail((prefix + ".k").c_str());
        B.n = (uint32_t)count;
        keep.push_back(raw);
        e = uploadRaw(B.k, keep.back().data(), raw.size(), s);
        if (e != cudaSuccess)
            return VFB_OK;
        // the entries' node locations, once (the BC launches read them instead of the neighbour chain)
        if (B.n) {
            e = B.locations.allocate(8ull * B.n * sizeof(uint32_t));
            if (e != cudaSuccess)
                return VFB_OK;
            if (const int rc = vfb_bc_locations(static_cast<const int32_t*>(B.k.ptr), B.n,
                                                static_cast<const uint32_t*>(L.nX.ptr),
                                                static_cast<const uint32_t*>(L.nY.ptr),
                                                static_cast<const uint32_t*>(L.nZ.ptr),
                                                static_cast<uint32_t*>(B.locations.ptr), s))
                return rc;
        }
        if (!need((prefix + ".q").c_str(), 8) || (unsigned long long)count != 27ull * B.n)
            return fail((prefix + ".q").c_str());
        e = uploadReal(B.q, raw, storage, s, keep);
        if (velocity) {
            const char* v[3] = { ".vx", ".vy", ".vz" };
            DeviceBuffer* vb[3] = { &B.vx, &B.vy, &B.vz };
            for (int i = 0; i < 3 && e == cudaSuccess; ++i) {
                if (!need((prefix + v[i]).c_str(), 8) || (uint32_t)count != B.n)
                    return fail((prefix + v[i]).c_str());
                e = uploadReal(*vb[i], raw, storage, s, keep, divisor);
            }
        }
        return VFB_OK;
    };
    if (e == cudaSuccess)
        if (const int rc = list("velocity", L.velocity, true))
            return rc;
    if (e == cudaSuccess)
        if (const int rc = list("slip", L.slip, false))
            return rc;
    if (e == cudaSuccess) {
        // a velocity on the geometry (setVelocityBoundaryCondition(GEOMETRY, ...)) comes with the list
        std::vector<char> probe;
        long long pc = 0;
        int pes = 0;
        const bool geometryVelocity = gridArray(grid, level, "geometry.vx", probe, pc, pes);
        if (const int rc = list("geometry", L.geometry, geometryVelocity, geometryVelocityDivisor))
            return rc;
    }
    // the stress lists (GridGenerator.cpp:319-341, which keeps a list only
    // when it has more than one entry) with the wall model's state, zero at start
    if (e == cudaSuccess && need("stress.k", 4) && count > 1) {
        StressListDevice& T = L.stress;
        T.n = (uint32_t)count;
        keep.push_back(raw);
        e = uploadRaw(T.k, keep.back().data(), raw.size(), s);
        if (e == cudaSuccess) {
            if (!need("stress.kN", 4) || (uint32_t)count != T.n)
                return fail("stress.kN");
            keep.push_back(raw);
            e = uploadRaw(T.kN, keep.back().data(), raw.size(), s);
        }
        if (e == cudaSuccess) {
            if (!need("stress.samplingOffset", 4) || (uint32_t)count != T.n)
                return fail("stress.samplingOffset");
            keep.push_back(raw);
            e = uploadRaw(T.samplingOffset, keep.back().data(), raw.size(), s);
        }
        if (e == cudaSuccess) {
            if (!need("stress.q", 8) || (unsigned long long)count != 27ull * T.n)
                return fail("stress.q");
            e = uploadReal(T.q, raw, storage, s, keep);
        }
        const char* reals[4] = { "stress.nx", "stress.ny", "stress.nz", "stress.z0" };
        DeviceBuffer* rb[4] = { &T.nx, &T.ny, &T.nz, &T.z0 };
        for (int i = 0; i < 4 && e == cudaSuccess; ++i) {
            if (!need(reals[i], 8) || (uint32_t)count != T.n)
                return fail(reals[i]);
            e = uploadReal(*rb[i], raw, storage, s, keep);
        }
        const size_t rbytes = (size_t)T.n * (computeIsDouble(storage) ? sizeof(double) : sizeof(float));
        for (int c = 0; c < 3 && e == cudaSuccess; ++c) {
            e = T.el[c].allocate(rbytes);
            if (e == cudaSuccess)
                e = cudaMemsetAsync(T.el[c].ptr, 0, rbytes, s);
            if (e == cudaSuccess)
                e = T.wm[c].allocate(rbytes);
            if (e == cudaSuccess)
                e = cudaMemsetAsync(T.wm[c].ptr, 0, rbytes, s);
        }
        if (e == cudaSuccess)
            e = T.locations.allocate(8ull * T.n * sizeof(uint32_t));
        if (e == cudaSuccess)
            if (const int rc = vfb_bc_locations(static_cast<const int32_t*>(T.k.ptr), T.n,
                                                static_cast<const uint32_t*>(L.nX.ptr),
                                                static_cast<const uint32_t*>(L.nY.ptr),
                                                static_cast<const uint32_t*>(L.nZ.ptr),
                                                static_cast<uint32_t*>(T.locations.ptr), s))
                return rc;
    }
    if (e == cudaSuccess && need("pressure.count", 4) && count == 1) {
        const int np = *reinterpret_cast<const int32_t*>(raw.data());
        for (int i = 0; i < np && e == cudaSuccess; ++i) {
            auto* P = new PressureListDevice;
            L.pressure.push_back(P);
            const std::string p = "pressure" + std::to_string(i);
            if (!need((p + ".k").c_str(), 4))
                return fail((p + ".k").c_str());
            P->n = (uint32_t)count;
            keep.push_back(raw);
            e = uploadRaw(P->k, keep.back().data(), raw.size(), s);
            if (e == cudaSuccess) {
                if (!need((p + ".kN").c_str(), 4) || (uint32_t)count != P->n)
                    return fail((p + ".kN").c_str());
                keep.push_back(raw);
                e = uploadRaw(P->kN, keep.back().data(), raw.size(), s);
            }
            if (e == cudaSuccess) {
                if (!need((p + ".rho").c_str(), 8) || (uint32_t)count != P->n)
                    return fail((p + ".rho").c_str());
                e = uploadReal(P->rho, raw, storage, s, keep);
            }
            if (e == cudaSuccess && P->n) {
                e = P->locations.allocate(16ull * P->n * sizeof(uint32_t));
                for (int half = 0; half < 2 && e == cudaSuccess; ++half)
                    if (const int rc = vfb_bc_locations(static_cast<const int32_t*>(half ? P->kN.ptr : P->k.ptr), P->n,
                                                        static_cast<const uint32_t*>(L.nX.ptr),
                                                        static_cast<const uint32_t*>(L.nY.ptr),
                                                        static_cast<const uint32_t*>(L.nZ.ptr),
                                                        static_cast<uint32_t*>(P->locations.ptr) + 8ull * P->n * half,
                                                        s))
                        return rc;
            }
            if (e == cudaSuccess) {
                if (!need((p + ".dir").c_str(), 4) || count != 1)
                    return fail((p + ".dir").c_str());
                P->direction = *reinterpret_cast<const int32_t*>(raw.data());
            }
        }
    }
    // interface cells to the next finer level, when the grid has them
    auto interface = [&](const char* tag, InterfaceDevice& I) -> int {
        const std::string t = tag;
        if (!need((t + ".coarse").c_str(), 4))
            return VFB_OK;
        I.n = (uint32_t)count;
        keep.push_back(raw);
        e = uploadRaw(I.coarse, keep.back().data(), raw.size(), s);
        if (e == cudaSuccess) {
            if (!need((t + ".fine").c_str(), 4) || (uint32_t)count != I.n)
                return fail((t + ".fine").c_str());
            keep.push_back(raw);
            e = uploadRaw(I.fine, keep.back().data(), raw.size(), s);
        }
        const char* off[3] = { ".offX", ".offY", ".offZ" };
        DeviceBuffer* ob[3] = { &I.offX, &I.offY, &I.offZ };
        for (int i = 0; i < 3 && e == cudaSuccess; ++i) {
            if (!need((t + off[i]).c_str(), 8) || (uint32_t)count != I.n)
                return fail((t + off[i]).c_str());
            e = uploadReal(*ob[i], raw, storage, s, keep);
        }
        return VFB_OK;
    };
    if (e == cudaSuccess)
        if (const int rc = interface("cf", L.coarseToFine))
            return rc;
    if (e == cudaSuccess)
        if (const int rc = interface("fc", L.fineToCoarse))
            return rc;
    if (e == cudaSuccess)
        e = L.dist.allocate(27ull * L.N * (size_t)elementBytes(storage));
    if (e == cudaSuccess)
        e = cudaMemsetAsync(L.dist.ptr, 0, L.dist.bytes, s);
    if (e != cudaSuccess)
        return setError(VFB_ERR_CUDA, "grid level %d: device upload failed: %s", level, cudaGetErrorString(e));
    return VFB_OK;
}

} // namespace
} // namespace vfb

namespace vfb
{
namespace
{

vfb_collision_args collisionArgs(const vfb_simulation& S, const Level& L)
{
    vfb_collision_args a;
    std::memset(&a, 0, sizeof(a));
    a.distributions = L.dist.ptr;
    a.numberOfLBnodes = L.N;
    a.neighborX = static_cast<const uint32_t*>(L.nX.ptr);
    a.neighborY = static_cast<const uint32_t*>(L.nY.ptr);
    a.neighborZ = static_cast<const uint32_t*>(L.nZ.ptr);
    a.fluidNodeIndices = static_cast<const uint32_t*>(L.fluid.ptr);
    a.numberOfFluidNodes = L.nFluid;
    a.omega = L.omega;
    for (int i = 0; i < 3; ++i) {
        a.forces[i] = S.params.forces[i];
        a.quadricLimiters[i] = S.params.quadricLimiters[i];
    }
    a.forceFactor = L.forceFactor;
    a.isEvenTimestep = L.isEven ? 1 : 0;
    a.collisionTemplate = VFB_TEMPLATE_DEFAULT;
    return a;
}

vfb_bc_lattice bcLattice(const Level& L)
{
    vfb_bc_lattice t;
    t.distributions = L.dist.ptr;
    t.numberOfLBnodes = L.N;
    t.neighborX = static_cast<const uint32_t*>(L.nX.ptr);
    t.neighborY = static_cast<const uint32_t*>(L.nY.ptr);
    t.neighborZ = static_cast<const uint32_t*>(L.nZ.ptr);
    t.omega = L.omega;
    t.isEvenTimestep = L.isEven ? 1 : 0;
    return t;
}

vfb_bc_list bcList(const BcListDevice& B)
{
    vfb_bc_list l;
    l.k = static_cast<const int32_t*>(B.k.ptr);
    l.q = B.q.ptr;
    l.Vx = B.vx.ptr;
    l.Vy = B.vy.ptr;
    l.Vz = B.vz.ptr;
    l.numberOfBCnodes = B.n;
    l.locations = static_cast<const uint32_t*>(B.locations.ptr);
    return l;
}

// CollisionStrategy (CollisisionStrategy.cpp:67-98): the fluid-node list of the level
int collision(vfb_simulation& S, Level& L, void* stream)
{
    vfb_collision_args a = collisionArgs(S, L);
    const bool k17 = S.params.collisionKernel == 0;
    if (L.plan)
        return k17 ? vfb_k17_collision_planned(L.plan, &a, stream) : vfb_bgk_collision_planned(L.plan, &a, stream);
    return k17 ? vfb_k17_collision(S.params.storage, &a, stream) : vfb_bgk_collision(S.params.storage, &a, stream);
}

// the entries `index` of a list, gathered on the host into a new device list
// (element sizes: k and locations 4 bytes, q and velocities `real` bytes)
int gatherList(const BcListDevice& B, const std::vector<uint32_t>& index, size_t real, BcListDevice& out,
               cudaStream_t s)
{
    const uint32_t n = B.n, m = (uint32_t)index.size();
    out.n = m;
    std::vector<char> k(4ull * n), loc(32ull * n), q(27ull * n * real), v[3];
    cudaError_t e = cudaMemcpyAsync(k.data(), B.k.ptr, k.size(), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(loc.data(), B.locations.ptr, loc.size(), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(q.data(), B.q.ptr, q.size(), cudaMemcpyDeviceToHost, s);
    const DeviceBuffer* vb[3] = { &B.vx, &B.vy, &B.vz };
    for (int c = 0; c < 3 && e == cudaSuccess; ++c)
        if (vb[c]->ptr) {
            v[c].resize(real * n);
            e = cudaMemcpyAsync(v[c].data(), vb[c]->ptr, v[c].size(), cudaMemcpyDeviceToHost, s);
        }
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return setError(VFB_ERR_CUDA, "residual BC list: %s", cudaGetErrorString(e));
    std::vector<char> k2(4ull * m), loc2(32ull * m), q2(27ull * m * real), v2[3];
    for (uint32_t j = 0; j < m; ++j) {
        const uint32_t i = index[j];
        std::memcpy(&k2[4ull * j], &k[4ull * i], 4);
        for (int l = 0; l < 8; ++l)
            std::memcpy(&loc2[4ull * ((size_t)l * m + j)], &loc[4ull * ((size_t)l * n + i)], 4);
        for (int d = 0; d < 27; ++d)
            std::memcpy(&q2[real * ((size_t)d * m + j)], &q[real * ((size_t)d * n + i)], real);
    }
    DeviceBuffer* ob[3] = { &out.vx, &out.vy, &out.vz };
    for (int c = 0; c < 3; ++c)
        if (!v[c].empty()) {
            v2[c].resize(real * m);
            for (uint32_t j = 0; j < m; ++j)
                std::memcpy(&v2[c][real * j], &v[c][real * index[j]], real);
        }
    e = uploadRaw(out.k, k2.data(), k2.size(), s);
    if (e == cudaSuccess)
        e = uploadRaw(out.locations, loc2.data(), loc2.size(), s);
    if (e == cudaSuccess)
        e = uploadRaw(out.q, q2.data(), q2.size(), s);
    for (int c = 0; c < 3 && e == cudaSuccess; ++c)
        if (!v2[c].empty())
            e = uploadRaw(*ob[c], v2[c].data(), v2[c].size(), s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return setError(VFB_ERR_CUDA, "residual BC list upload: %s", cudaGetErrorString(e));
    return VFB_OK;
}

// the plan's BC epilogue for a level: the post-collision lists in schedule
// order (a stress list's nodes excluded, since its kernel runs between them),
// then the residual lists of the entries the epilogue does not take
int setupEpilogue(vfb_simulation& S, Level& L, cudaStream_t s)
{
    const vfb_sim_params& P = S.params;
    BcListDevice* full[4] = { &L.velocity, &L.noSlip, &L.slip, &L.geometry };
    const int kinds[4] = { P.velocityBC, P.noSlipBC, P.slipBC, P.geometryBC };
    vfb_bc_epilogue_list lists[4];
    int which[4];
    int n = 0;
    DeviceBuffer fused[4];
    for (int i = 0; i < 4; ++i) {
        if (full[i]->n == 0 || kinds[i] < 0)
            continue;
        if (fused[n].allocate(full[i]->n) != cudaSuccess)
            return setError(VFB_ERR_CUDA, "epilogue flags");
        vfb_bc_epilogue_list& e = lists[n];
        e.kind = kinds[i];
        e.k = static_cast<const int32_t*>(full[i]->k.ptr);
        e.q = full[i]->q.ptr;
        e.Vx = full[i]->vx.ptr;
        e.Vy = full[i]->vy.ptr;
        e.Vz = full[i]->vz.ptr;
        e.locations = static_cast<const uint32_t*>(full[i]->locations.ptr);
        e.numberOfBCnodes = full[i]->n;
        e.fused = static_cast<uint8_t*>(fused[n].ptr);
        which[n++] = i;
    }
    if (n == 0)
        return VFB_OK;
    const bool stress = L.stress.n > 0 && P.stressBC >= 0;
    const int rc = vfb_collision_plan_set_bc_epilogue(L.plan, lists, n, L.omega,
                                                      stress ? static_cast<const int32_t*>(L.stress.k.ptr) : nullptr,
                                                      stress ? L.stress.n : 0u, s);
    if (rc == VFB_ERR_UNSUPPORTED) { // a tuning configuration without the epilogue: separate launches
        clearError();
        return VFB_OK;
    }
    if (rc)
        return rc;
    const size_t real = computeIsDouble(P.storage) ? sizeof(double) : sizeof(float);
    for (int j = 0; j < n; ++j) {
        const int i = which[j];
        std::vector<uint8_t> f(full[i]->n);
        if (cudaMemcpyAsync(f.data(), fused[j].ptr, f.size(), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return setError(VFB_ERR_CUDA, "epilogue flags: %s", cudaGetErrorString(cudaGetLastError()));
        ResidualList& R = L.residual[i];
        R.index.clear();
        for (uint32_t e = 0; e < full[i]->n; ++e)
            if (!f[e])
                R.index.push_back(e);
        if (const int g = gatherList(*full[i], R.index, real, R.list, s))
            return g;
    }
    // lists the epilogue was not given keep all their entries
    for (int i = 0; i < 4; ++i) {
        bool given = false;
        for (int j = 0; j < n; ++j)
            given = given || which[j] == i;
        if (!given && full[i]->n) {
            ResidualList& R = L.residual[i];
            R.index.resize(full[i]->n);
            for (uint32_t e = 0; e < full[i]->n; ++e)
                R.index[e] = e;
            if (const int g = gatherList(*full[i], R.index, real, R.list, s))
                return g;
        }
    }
    L.epilogue = true;
    return VFB_OK;
}

vfb_stress_list stressList(StressListDevice& T, bool monitor)
{
    vfb_stress_list l;
    std::memset(&l, 0, sizeof(l));
    l.k = static_cast<const int32_t*>(T.k.ptr);
    l.kN = static_cast<const int32_t*>(T.kN.ptr);
    l.q = T.q.ptr;
    l.normalX = T.nx.ptr;
    l.normalY = T.ny.ptr;
    l.normalZ = T.nz.ptr;
    l.Vx = T.el[0].ptr;
    l.Vy = T.el[1].ptr;
    l.Vz = T.el[2].ptr;
    l.Vx1 = T.wm[0].ptr;
    l.Vy1 = T.wm[1].ptr;
    l.Vz1 = T.wm[2].ptr;
    l.samplingOffset = static_cast<const int32_t*>(T.samplingOffset.ptr);
    l.z0 = T.z0.ptr;
    if (monitor) {
        l.uStar = T.uStar.ptr;
        l.Fx = T.F[0].ptr;
        l.Fy = T.F[1].ptr;
        l.Fz = T.F[2].ptr;
    }
    l.numberOfBCnodes = T.n;
    l.locations = static_cast<const uint32_t*>(T.locations.ptr);
    return l;
}

// UpdateGrid27::postCollisionBC (UpdateGrid27.cpp:228-263): velocity, no-slip,
// slip, stress, geometry; every kernel only when its list is not empty
int postCollisionBC(vfb_simulation& S, Level& L, void* stream)
{
    const vfb_bc_lattice t = bcLattice(L);
    const int storage = S.params.storage;
    struct Item {
        const BcListDevice* list;
        int kind;
    } items[4] = { { L.epilogue ? &L.residual[0].list : &L.velocity, S.params.velocityBC },
                   { L.epilogue ? &L.residual[1].list : &L.noSlip, S.params.noSlipBC },
                   { L.epilogue ? &L.residual[2].list : &L.slip, S.params.slipBC },
                   { L.epilogue ? &L.residual[3].list : &L.geometry, S.params.geometryBC } };
    for (int i = 0; i < 4; ++i) {
        const Item& it = items[i];
        if (i == 3 && L.stress.n > 0 && S.params.stressBC >= 0) {
            // runStressWallModelKernelPost (BoundaryConditionKernelManager.cpp:330-334);
            // the launchers of Stress.cu:42-160 pass the level's velocityY as vz too
            if (!L.fields[1].ptr || !L.fields[2].ptr)
                return setError(VFB_ERR_CONFIGURATION,
                                "the stress BC reads the level's macroscopic velocity: initialise the level first");
            const vfb_stress_list l = stressList(L.stress, S.params.hasWallModelMonitor != 0);
            if (const int rc = vfb_bc_stress(S.params.stressBC, storage, &t, &l, nullptr, L.fields[1].ptr,
                                             L.fields[2].ptr, L.fields[2].ptr, stream))
                return rc;
        }
        if (it.list->n == 0 || it.kind < 0)
            continue;
        const vfb_bc_list l = bcList(*it.list);
        if (const int rc = vfb_bc_post(it.kind, storage, &t, &l, stream))
            return rc;
    }
    return VFB_OK;
}

// UpdateGrid27::preCollisionBC (UpdateGrid27.cpp:289-308): the pressure lists
int preCollisionBC(vfb_simulation& S, Level& L, void* stream)
{
    if (S.params.pressureBC < 0)
        return VFB_OK;
    const vfb_bc_lattice t = bcLattice(L);
    for (const PressureListDevice* P : L.pressure) {
        if (P->n == 0)
            continue;
        const auto* k = static_cast<const int32_t*>(P->k.ptr);
        const auto* kN = static_cast<const int32_t*>(P->kN.ptr);
        // BoundaryConditionFactory::getPressureBoundaryConditionPre (BoundaryConditionFactory.cpp:151-168)
        const int rc = S.params.pressureBC == 0
                           ? pressureNoneqWithLocations(S.params.storage, &t, k, kN, P->rho.ptr, P->n, P->direction,
                                                        static_cast<const uint32_t*>(P->locations.ptr), stream)
                           : vfb_bc_outflow_nonreflecting(S.params.storage, &t, k, kN, P->n, P->direction,
                                                          S.params.pressureBC == 2,
                                                          S.params.outflowPressureCorrectionFactor, stream);
        if (rc)
            return rc;
    }
    return VFB_OK;
}

// GridScalingKernelManager::runFineToCoarseKernelLB / runCoarseToFineKernelLB
// (GridScalingKernelManager.cpp:64-74), in the order of Refinement_noExchange
// (RefinementStrategy.cpp:169-178): fine to coarse, then coarse to fine
int refinement(vfb_simulation& S, Level& C, Level& F, void* stream)
{
    vfb_scaling_args a;
    std::memset(&a, 0, sizeof(a));
    a.distributionsCoarse = C.dist.ptr;
    a.distributionsFine = F.dist.ptr;
    a.neighborXcoarse = static_cast<const uint32_t*>(C.nX.ptr);
    a.neighborYcoarse = static_cast<const uint32_t*>(C.nY.ptr);
    a.neighborZcoarse = static_cast<const uint32_t*>(C.nZ.ptr);
    a.neighborXfine = static_cast<const uint32_t*>(F.nX.ptr);
    a.neighborYfine = static_cast<const uint32_t*>(F.nY.ptr);
    a.neighborZfine = static_cast<const uint32_t*>(F.nZ.ptr);
    a.numberOfLBnodesCoarse = C.N;
    a.numberOfLBnodesFine = F.N;
    a.isEvenTimestep = C.isEven ? 1 : 0;
    a.omegaCoarse = C.omega;
    a.omegaFine = F.omega;
    const InterfaceDevice* order[2] = { &C.fineToCoarse, &C.coarseToFine };
    if (C.interfaceTogether && C.fineToCoarse.n && C.coarseToFine.n) {
        vfb_scaling_args b[2] = { a, a };
        for (int i = 0; i < 2; ++i) {
            const InterfaceDevice& I = *order[i];
            b[i].coarseCells = static_cast<const uint32_t*>(I.coarse.ptr);
            b[i].fineCells = static_cast<const uint32_t*>(I.fine.ptr);
            b[i].numberOfCells = I.n;
            b[i].offsetX = I.offX.ptr;
            b[i].offsetY = I.offY.ptr;
            b[i].offsetZ = I.offZ.ptr;
            b[i].fineWriteMask = static_cast<const uint8_t*>(I.mask.ptr);
            b[i].coarseBlocks = static_cast<const uint32_t*>(I.blocksC.ptr);
            b[i].fineBlocks = static_cast<const uint32_t*>(I.blocksF.ptr);
        }
        return vfb_scale_interface(S.params.storage, &b[0], &b[1], stream);
    }
    for (int i = 0; i < 2; ++i) {
        const InterfaceDevice& I = *order[i];
        if (I.n == 0)
            continue;
        a.coarseCells = static_cast<const uint32_t*>(I.coarse.ptr);
        a.fineCells = static_cast<const uint32_t*>(I.fine.ptr);
        a.numberOfCells = I.n;
        a.offsetX = I.offX.ptr;
        a.offsetY = I.offY.ptr;
        a.offsetZ = I.offZ.ptr;
        a.fineWriteMask = static_cast<const uint8_t*>(I.mask.ptr);
        a.coarseBlocks = static_cast<const uint32_t*>(I.blocksC.ptr);
        a.fineBlocks = static_cast<const uint32_t*>(I.blocksF.ptr);
        const int rc = i == 0 ? vfb_scale_fine_to_coarse(S.params.storage, &a, stream)
                              : vfb_scale_coarse_to_fine(S.params.storage, &a, stream);
        if (rc)
            return rc;
    }
    return VFB_OK;
}

// UpdateGrid27::updateGrid (UpdateGrid27.cpp:54-96).  The reference runs the
// finer level's two substeps, then this level's collision, BCs and parity
// swap, then fine-to-coarse and coarse-to-fine.  The finer level's substeps
// touch only the finer level's arrays and this level's step only this
// level's, and both read what the previous refinement wrote, so they run
// side by side here: the substeps on this level's side stream, forked from
// and joined back into the level's stream before the refinement.  Every
// array sees the reference's sequence of writes, so the result is the same;
// the short BC and interface launches of one level overlap the other's work.
int updateGrid(vfb_simulation& S, int level, void* stream)
{
    const int finest = (int)S.levels.size() - 1;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc = VFB_OK;
    if (level != finest) {
        cudaStream_t side = S.side[level];
        if (cudaEventRecord(S.fork[level], s) != cudaSuccess || cudaStreamWaitEvent(side, S.fork[level], 0) != cudaSuccess)
            return setError(VFB_ERR_CUDA, "level fork: %s", cudaGetErrorString(cudaGetLastError()));
        rc = updateGrid(S, level + 1, side);
        if (rc == VFB_OK)
            rc = updateGrid(S, level + 1, side);
        // joined below in every case, so that no side stream is left forked
        if (cudaEventRecord(S.join[level], side) != cudaSuccess && rc == VFB_OK)
            rc = setError(VFB_ERR_CUDA, "level join: %s", cudaGetErrorString(cudaGetLastError()));
    }
    Level& L = *S.levels[level];
    if (rc == VFB_OK)
        rc = collision(S, L, stream);
    if (rc == VFB_OK)
        rc = postCollisionBC(S, L, stream);
    if (rc == VFB_OK) {
        L.isEven = !L.isEven; // swapBetweenEvenAndOddTimestep (:265-269)
        rc = preCollisionBC(S, L, stream);
    }
    if (level == finest)
        return rc;
    if (cudaStreamWaitEvent(s, S.join[level], 0) != cudaSuccess && rc == VFB_OK)
        rc = setError(VFB_ERR_CUDA, "level join: %s", cudaGetErrorString(cudaGetLastError()));
    if (rc != VFB_OK)
        return rc;
    return refinement(S, L, *S.levels[level + 1], stream);
}

bool validKind(int k, int lo, int hi) { return k < 0 || (k >= lo && k <= hi); }

} // namespace
} // namespace vfb

using namespace vfb;

extern "C" int vfb_sim_create(const vfb_sim_params* params, void* grid, vfb_simulation** sim, void* stream)
{
    clearError();
    if (!params || !grid || !sim)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    *sim = nullptr;
    const vfb_sim_params& P = *params;
    if (elementBytes(P.storage) == 0)
        return setError(VFB_ERR_INVALID_ARGUMENT, "unknown storage %d", P.storage);
    if (P.collisionKernel != 0 && P.collisionKernel != 1)
        return setError(VFB_ERR_INVALID_ARGUMENT, "unknown collision kernel %d", P.collisionKernel);
    if (P.velocityBC != VFB_BC_VELOCITY_INTERPOLATED && P.velocityBC != VFB_BC_VELOCITY_BOUNCE_BACK &&
        P.velocityBC != VFB_BC_VELOCITY_WITH_PRESSURE)
        return setError(VFB_ERR_INVALID_ARGUMENT, "velocityBC must be a velocity kind");
    if (!validKind(P.noSlipBC, VFB_BC_NOSLIP_INTERPOLATED, VFB_BC_NOSLIP_BOUNCE_BACK) ||
        !(validKind(P.geometryBC, VFB_BC_NOSLIP_INTERPOLATED, VFB_BC_NOSLIP_BOUNCE_BACK) ||
          P.geometryBC == VFB_BC_VELOCITY_INTERPOLATED || P.geometryBC == VFB_BC_VELOCITY_BOUNCE_BACK ||
          P.geometryBC == VFB_BC_VELOCITY_WITH_PRESSURE) ||
        !(P.slipBC < 0 || P.slipBC == VFB_BC_SLIP) || !(P.pressureBC >= -1 && P.pressureBC <= 2) ||
        !validKind(P.stressBC, VFB_BC_STRESS_INTERPOLATED, VFB_BC_STRESS_BOUNCE_BACK_PRESSURE))
        return setError(VFB_ERR_INVALID_ARGUMENT, "invalid boundary-condition selection");
    if (!(P.viscosity > 0.0))
        return setError(VFB_ERR_INVALID_ARGUMENT, "viscosity %g must be positive", P.viscosity);
    const int nLevels = vfb_grid_levels(grid);
    if (nLevels < 1)
        return setError(VFB_ERR_INVALID_ARGUMENT, "grid has no level");
    auto* S = new vfb_simulation;
    S->params = P;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    std::vector<std::vector<char>> keep;
    int rc = VFB_OK;
    for (int l = 0; l < nLevels && rc == VFB_OK; ++l) {
        auto* L = new Level;
        S->levels.push_back(L);
        rc = uploadLevel(*L, grid, l, P.storage, P.velocityRatio > 0.0 ? P.velocityRatio : 1.0, s, keep);
        if (rc == VFB_OK && P.hasWallModelMonitor && L->stress.n > 0) {
            // CudaMemoryManager::cudaAllocWallModel with the monitor
            const size_t rbytes = (size_t)L->stress.n * (computeIsDouble(P.storage) ? sizeof(double) : sizeof(float));
            DeviceBuffer* mon[4] = { &L->stress.uStar, &L->stress.F[0], &L->stress.F[1], &L->stress.F[2] };
            for (DeviceBuffer* b : mon)
                if (rc == VFB_OK &&
                    (b->allocate(rbytes) != cudaSuccess || cudaMemsetAsync(b->ptr, 0, rbytes, s) != cudaSuccess))
                    rc = setError(VFB_ERR_CUDA, "wall-model monitor allocation failed");
        }
        if (rc == VFB_OK && P.geometryBC >= VFB_BC_VELOCITY_INTERPOLATED && L->geometry.n > 0 && !L->geometry.vx.ptr)
            rc = setError(VFB_ERR_CONFIGURATION, "a velocity geometry BC needs the geometry velocities (level %d)", l);
        if (rc == VFB_OK) {
            // the inverse neighbour: required by useInitNeq, otherwise uploaded when the grid has it
            std::vector<char> nn;
            long long count = 0;
            int es = 0;
            if (!gridArray(grid, l, "neighborNeg", nn, count, es) || es != 4 || (unsigned long long)count != L->N) {
                if (P.useInitNeq)
                    rc = setError(VFB_ERR_CONFIGURATION, "grid level %d: array neighborNeg (needed by useInitNeq)", l);
            } else {
                keep.push_back(std::move(nn));
                if (uploadRaw(L->nNeg, keep.back().data(), keep.back().size(), s) != cudaSuccess)
                    rc = setError(VFB_ERR_CUDA, "neighborNeg upload failed");
            }
        }
        // Parameter::initLBMSimulationParameter (Parameter.cpp:395-420)
        const double nu = P.viscosity * std::pow(2.0, l);
        L->omega = 1.0 / (3.0 * nu + 0.5);
        L->forceFactor = 1.0 / std::pow(2.0, l);
    }
    // a side stream and fork / join events per level with a finer level
    for (int l = 0; l + 1 < nLevels && rc == VFB_OK; ++l) {
        cudaStream_t side = nullptr;
        cudaEvent_t f = nullptr, j = nullptr;
        if (cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&f, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&j, cudaEventDisableTiming) != cudaSuccess)
            rc = setError(VFB_ERR_CUDA, "level streams: %s", cudaGetErrorString(cudaGetLastError()));
        if (side)
            S->side.push_back(side);
        if (f)
            S->fork.push_back(f);
        if (j)
            S->join.push_back(j);
    }
    // the kinetic-energy analyzer's node set of every level (KineticEnergyAnalyzer.cu:137-154)
    for (int l = 0; l < nLevels && rc == VFB_OK; ++l) {
        std::vector<char> geo, nx, ny, nz, nn;
        long long count = 0;
        int es = 0;
        if (!gridArray(grid, l, "geo", geo, count, es) || !gridArray(grid, l, "neighborX", nx, count, es) ||
            !gridArray(grid, l, "neighborY", ny, count, es) || !gridArray(grid, l, "neighborZ", nz, count, es))
            continue;
        const bool haveInverse = gridArray(grid, l, "neighborNeg", nn, count, es) && es == 4;
        if (!haveInverse)
            continue;
        const uint32_t* G = reinterpret_cast<const uint32_t*>(geo.data());
        const uint32_t* X = reinterpret_cast<const uint32_t*>(nx.data());
        const uint32_t* Y = reinterpret_cast<const uint32_t*>(ny.data());
        const uint32_t* Z = reinterpret_cast<const uint32_t*>(nz.data());
        const uint32_t* W = reinterpret_cast<const uint32_t*>(nn.data());
        const uint64_t N = S->levels[l]->N;
        auto fluid = [&](uint32_t k) { return k < N && G[k] == VFB_GEO_FLUID; };
        keep.emplace_back();
        std::vector<char>& list = keep.back();
        for (uint64_t k = 0; k < N; ++k) {
            if (!fluid((uint32_t)k))
                continue;
            const uint32_t w = W[k];
            if (!fluid(X[k]) || !fluid(Y[k]) || !fluid(Z[k]) || !fluid(w))
                continue;
            if (!fluid(Z[Y[w]]) || !fluid(Z[X[w]]) || !fluid(Y[X[w]]))
                continue;
            const uint32_t v = (uint32_t)k;
            list.insert(list.end(), reinterpret_cast<const char*>(&v), reinterpret_cast<const char*>(&v) + 4);
        }
        S->levels[l]->nEnergy = (uint32_t)(list.size() / 4);
        if (uploadRaw(S->levels[l]->energyNodes, list.data(), list.size(), s) != cudaSuccess)
            rc = setError(VFB_ERR_CUDA, "energy node upload failed");
    }
    // coarse-to-fine cells that share fine nodes: one writer per node (the last in list order)
    for (int l = 0; l + 1 < nLevels && rc == VFB_OK; ++l) {
        Level& C = *S->levels[l];
        if (C.coarseToFine.n == 0)
            continue;
        std::vector<char> cells, nx, ny, nz;
        long long count = 0;
        int es = 0;
        if (!gridArray(grid, l, "cf.fine", cells, count, es) || !gridArray(grid, l + 1, "neighborX", nx, count, es) ||
            !gridArray(grid, l + 1, "neighborY", ny, count, es) || !gridArray(grid, l + 1, "neighborZ", nz, count, es)) {
            rc = setError(VFB_ERR_CONFIGURATION, "grid level %d: interface arrays", l);
            break;
        }
        keep.emplace_back(27 * (size_t)C.coarseToFine.n);
        std::vector<char>& mask = keep.back();
        rc = vfb_scaling_write_mask(reinterpret_cast<const uint32_t*>(cells.data()), C.coarseToFine.n,
                                    reinterpret_cast<const uint32_t*>(nx.data()),
                                    reinterpret_cast<const uint32_t*>(ny.data()),
                                    reinterpret_cast<const uint32_t*>(nz.data()), S->levels[l + 1]->N,
                                    reinterpret_cast<uint8_t*>(mask.data()));
        if (rc == VFB_OK && uploadRaw(C.coarseToFine.mask, mask.data(), mask.size(), s) != cudaSuccess)
            rc = setError(VFB_ERR_CUDA, "interface mask upload failed");
        // whether fine-to-coarse and coarse-to-fine can share one launch
        std::vector<char> cfc, fcc, fcf, cnx, cny, cnz;
        if (rc == VFB_OK && C.fineToCoarse.n &&
            gridArray(grid, l, "cf.coarse", cfc, count, es) && gridArray(grid, l, "fc.coarse", fcc, count, es) &&
            gridArray(grid, l, "fc.fine", fcf, count, es) && gridArray(grid, l, "neighborX", cnx, count, es) &&
            gridArray(grid, l, "neighborY", cny, count, es) && gridArray(grid, l, "neighborZ", cnz, count, es)) {
            int together = 0;
            auto u32 = [](const std::vector<char>& v) { return reinterpret_cast<const uint32_t*>(v.data()); };
            rc = vfb_scaling_independent(u32(fcc), u32(fcf), C.fineToCoarse.n, u32(cfc), u32(cells),
                                         C.coarseToFine.n, reinterpret_cast<const uint8_t*>(mask.data()), u32(cnx),
                                         u32(cny), u32(cnz), C.N, u32(nx), u32(ny), u32(nz), S->levels[l + 1]->N,
                                         &together);
            C.interfaceTogether = together != 0;
        }
    }
    // the interface cells' blocks of node indices, walked once on the device
    for (int l = 0; l + 1 < nLevels && rc == VFB_OK; ++l) {
        Level& C = *S->levels[l];
        Level& F = *S->levels[l + 1];
        for (InterfaceDevice* I : { &C.coarseToFine, &C.fineToCoarse }) {
            if (I->n == 0)
                continue;
            if (I->blocksC.allocate(27ull * I->n * sizeof(uint32_t)) != cudaSuccess ||
                I->blocksF.allocate(27ull * I->n * sizeof(uint32_t)) != cudaSuccess) {
                rc = setError(VFB_ERR_CUDA, "interface block tables");
                break;
            }
            rc = vfb_scaling_blocks(static_cast<const uint32_t*>(I->coarse.ptr), I->n,
                                    static_cast<const uint32_t*>(C.nX.ptr), static_cast<const uint32_t*>(C.nY.ptr),
                                    static_cast<const uint32_t*>(C.nZ.ptr), static_cast<uint32_t*>(I->blocksC.ptr), s);
            if (rc == VFB_OK)
                rc = vfb_scaling_blocks(static_cast<const uint32_t*>(I->fine.ptr), I->n,
                                        static_cast<const uint32_t*>(F.nX.ptr), static_cast<const uint32_t*>(F.nY.ptr),
                                        static_cast<const uint32_t*>(F.nZ.ptr), static_cast<uint32_t*>(I->blocksF.ptr),
                                        s);
            if (rc != VFB_OK)
                break;
        }
    }
    if (rc == VFB_OK && cudaStreamSynchronize(s) != cudaSuccess)
        rc = setError(VFB_ERR_CUDA, "upload failed: %s", cudaGetErrorString(cudaGetLastError()));
    for (size_t l = 0; l < S->levels.size() && rc == VFB_OK && P.usePlan; ++l) {
        Level& L = *S->levels[l];
        vfb_collision_args a = collisionArgs(*S, L);
        rc = vfb_collision_plan_create(P.storage, &a, &L.plan, stream);
        if (rc == VFB_OK && P.bcEpilogue)
            rc = setupEpilogue(*S, L, s);
    }
    if (rc != VFB_OK) {
        delete S;
        return rc;
    }
    *sim = S;
    return VFB_OK;
}

extern "C" int vfb_sim_destroy(vfb_simulation* sim)
{
    clearError();
    delete sim;
    return VFB_OK;
}

extern "C" int vfb_sim_levels(const vfb_simulation* sim) { return sim ? (int)sim->levels.size() : 0; }

static Level* levelOf(vfb_simulation* sim, int level)
{
    if (!sim || level < 0 || level >= (int)sim->levels.size()) {
        setError(VFB_ERR_INVALID_ARGUMENT, "no level %d", level);
        return nullptr;
    }
    return sim->levels[level];
}

extern "C" int vfb_sim_init_level(vfb_simulation* sim, int level, const void* rho, const void* vx, const void* vy,
                                  const void* vz, void* stream)
{
    clearError();
    Level* L = levelOf(sim, level);
    if (!L)
        return VFB_ERR_INVALID_ARGUMENT;
    if (!rho || !vx || !vy || !vz)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL field");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t bytes = L->N * (computeIsDouble(sim->params.storage) ? sizeof(double) : sizeof(float));
    if (L->fieldBuffers(bytes) != cudaSuccess)
        return setError(VFB_ERR_CUDA, "field buffers: %s", cudaGetErrorString(cudaGetLastError()));
    DeviceBuffer* f = L->fields;
    const void* host[4] = { rho, vx, vy, vz };
    for (int i = 0; i < 4; ++i)
        if (cudaMemcpyAsync(f[i].ptr, host[i], bytes, cudaMemcpyHostToDevice, s) != cudaSuccess)
            return setError(VFB_ERR_CUDA, "field upload failed");
    int rc = VFB_OK;
    const auto* geo = static_cast<const uint32_t*>(L->geo.ptr);
    const auto* nX = static_cast<const uint32_t*>(L->nX.ptr);
    const auto* nY = static_cast<const uint32_t*>(L->nY.ptr);
    const auto* nZ = static_cast<const uint32_t*>(L->nZ.ptr);
    // InitNavierStokesCompressible::init (InitNavierStokesCompressible.cu:46-83)
    for (int even = 0; even < 2 && rc == VFB_OK; ++even) {
        if (sim->params.useInitNeq)
            rc = vfb_init_nonequilibrium(sim->params.storage, L->dist.ptr, L->N, geo, nX, nY, nZ,
                                         static_cast<const uint32_t*>(L->nNeg.ptr), f[0].ptr, f[1].ptr, f[2].ptr,
                                         f[3].ptr, L->omega, even, stream);
        else
            rc = vfb_init_equilibrium(sim->params.storage, L->dist.ptr, L->N, geo, nX, nY, nZ, f[0].ptr, f[1].ptr,
                                      f[2].ptr, f[3].ptr, even, stream);
    }
    L->isEven = true;
    // the caller may reuse its host arrays on return: wait for the copies and the init kernels
    if (cudaStreamSynchronize(s) != cudaSuccess && rc == VFB_OK)
        rc = setError(VFB_ERR_CUDA, "init failed: %s", cudaGetErrorString(cudaGetLastError()));
    return rc;
}

namespace
{
unsigned long long parityPattern(const vfb_simulation& S)
{
    unsigned long long key = 0;
    for (size_t l = 0; l < S.levels.size(); ++l)
        key |= (unsigned long long)(S.levels[l]->isEven ? 1 : 0) << l;
    return key;
}

// the graph of two coarse steps from the current parity pattern (captured on first use)
int graphForPattern(vfb_simulation& S, cudaGraphExec_t& exec)
{
    const unsigned long long key = parityPattern(S);
    auto it = S.graphs.find(key);
    if (it != S.graphs.end()) {
        exec = it->second;
        return VFB_OK;
    }
    if (!S.captureStream && cudaStreamCreateWithFlags(&S.captureStream, cudaStreamNonBlocking) != cudaSuccess)
        return setError(VFB_ERR_CUDA, "capture stream: %s", cudaGetErrorString(cudaGetLastError()));
    if (cudaStreamBeginCapture(S.captureStream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return setError(VFB_ERR_CUDA, "begin capture: %s", cudaGetErrorString(cudaGetLastError()));
    int rc = VFB_OK;
    for (int t = 0; t < 2 && rc == VFB_OK; ++t)
        rc = updateGrid(S, 0, S.captureStream);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(S.captureStream, &graph);
    // nothing ran: the parities are back to the pattern the capture started from
    // (two coarse steps flip every level an even number of times)
    if (rc == VFB_OK && (e != cudaSuccess || !graph))
        rc = setError(VFB_ERR_CUDA, "end capture: %s", cudaGetErrorString(e));
    if (rc == VFB_OK && parityPattern(S) != key)
        rc = setError(VFB_ERR_CONFIGURATION, "the parities did not return after two coarse steps");
    if (rc == VFB_OK && cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess)
        rc = setError(VFB_ERR_CUDA, "graph instantiation: %s", cudaGetErrorString(cudaGetLastError()));
    if (graph)
        cudaGraphDestroy(graph);
    if (rc == VFB_OK)
        S.graphs[key] = exec;
    return rc;
}
} // namespace

extern "C" int vfb_sim_run(vfb_simulation* sim, unsigned int steps, void* stream)
{
    clearError();
    if (!sim)
        return setError(VFB_ERR_INVALID_ARGUMENT, "sim is NULL");
    unsigned int t = 0;
    if (sim->params.useGraphs) {
        // two ordinary steps first: every kernel path has run once before a capture
        for (; t < steps && sim->stepsRun < 2; ++t, ++sim->stepsRun)
            if (const int rc = updateGrid(*sim, 0, stream))
                return rc;
        for (; t + 2 <= steps; t += 2) {
            cudaGraphExec_t exec = nullptr;
            if (const int rc = graphForPattern(*sim, exec))
                return rc;
            if (cudaGraphLaunch(exec, static_cast<cudaStream_t>(stream)) != cudaSuccess)
                return setError(VFB_ERR_CUDA, "graph launch: %s", cudaGetErrorString(cudaGetLastError()));
            sim->stepsRun += 2;
        }
    }
    for (; t < steps; ++t, ++sim->stepsRun)
        if (const int rc = updateGrid(*sim, 0, stream))
            return rc;
    return VFB_OK;
}

extern "C" int vfb_sim_macroscopic(vfb_simulation* sim, int level, void* rho, void* vx, void* vy, void* vz,
                                   void* stream)
{
    clearError();
    Level* L = levelOf(sim, level);
    if (!L)
        return VFB_ERR_INVALID_ARGUMENT;
    if (!rho || !vx || !vy || !vz)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL output");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t bytes = L->N * (computeIsDouble(sim->params.storage) ? sizeof(double) : sizeof(float));
    if (L->fieldBuffers(bytes) != cudaSuccess)
        return setError(VFB_ERR_CUDA, "field buffers: %s", cudaGetErrorString(cudaGetLastError()));
    DeviceBuffer* f = L->fields;
    int rc = vfb_macroscopic(sim->params.storage, L->dist.ptr, L->N, static_cast<const uint32_t*>(L->geo.ptr),
                             static_cast<const uint32_t*>(L->nX.ptr), static_cast<const uint32_t*>(L->nY.ptr),
                             static_cast<const uint32_t*>(L->nZ.ptr), L->isEven ? 1 : 0, f[0].ptr, f[1].ptr, f[2].ptr,
                             f[3].ptr, stream);
    void* out[4] = { rho, vx, vy, vz };
    for (int i = 0; i < 4 && rc == VFB_OK; ++i)
        if (cudaMemcpyAsync(out[i], f[i].ptr, bytes, cudaMemcpyDeviceToHost, s) != cudaSuccess)
            rc = setError(VFB_ERR_CUDA, "copy failed");
    if (cudaStreamSynchronize(s) != cudaSuccess && rc == VFB_OK)
        rc = setError(VFB_ERR_CUDA, "macroscopic failed: %s", cudaGetErrorString(cudaGetLastError()));
    return rc;
}

extern "C" int vfb_sim_mass_and_energy(vfb_simulation* sim, int level, double* out3, void* stream)
{
    clearError();
    Level* L = levelOf(sim, level);
    if (!L)
        return VFB_ERR_INVALID_ARGUMENT;
    return vfb_mass_and_energy(sim->params.storage, L->dist.ptr, L->N, static_cast<const uint32_t*>(L->nX.ptr),
                               static_cast<const uint32_t*>(L->nY.ptr), static_cast<const uint32_t*>(L->nZ.ptr),
                               static_cast<const uint32_t*>(L->fluid.ptr), L->nFluid, L->isEven ? 1 : 0, out3, stream);
}

extern "C" int vfb_sim_saturated_populations(vfb_simulation* sim, int level, unsigned long long* count, void* stream)
{
    clearError();
    Level* L = levelOf(sim, level);
    if (!L)
        return VFB_ERR_INVALID_ARGUMENT;
    return vfb_saturated_populations(sim->params.storage, L->dist.ptr, L->N, count, stream);
}

extern "C" int vfb_sim_enstrophy(vfb_simulation* sim, int level, double* out2, void* stream)
{
    clearError();
    Level* L = levelOf(sim, level);
    if (!L)
        return VFB_ERR_INVALID_ARGUMENT;
    if (!out2)
        return setError(VFB_ERR_INVALID_ARGUMENT, "out2 is NULL");
    if (!L->nNeg.ptr)
        return setError(VFB_ERR_CONFIGURATION, "level %d has no inverse neighbour array", level);
    const bool dbl = computeIsDouble(sim->params.storage);
    const size_t bytes = L->N * (dbl ? sizeof(double) : sizeof(float));
    DeviceBuffer m[4];
    for (auto& b : m)
        if (b.allocate(bytes) != cudaSuccess)
            return setError(VFB_ERR_CUDA, "macroscopic buffers");
    const auto* geo = static_cast<const uint32_t*>(L->geo.ptr);
    const auto* nX = static_cast<const uint32_t*>(L->nX.ptr);
    const auto* nY = static_cast<const uint32_t*>(L->nY.ptr);
    const auto* nZ = static_cast<const uint32_t*>(L->nZ.ptr);
    int rc = vfb_macroscopic(sim->params.storage, L->dist.ptr, L->N, geo, nX, nY, nZ, L->isEven ? 1 : 0, m[0].ptr,
                             m[1].ptr, m[2].ptr, m[3].ptr, stream);
    if (rc == VFB_OK)
        rc = vfb_enstrophy(dbl ? VFB_FP64 : VFB_FP32, m[0].ptr, m[1].ptr, m[2].ptr, m[3].ptr, L->N, geo, nX, nY, nZ,
                           static_cast<const uint32_t*>(L->nNeg.ptr), out2, stream);
    return rc;
}

// Simulation::readAndWriteFiles (Simulation.cpp:595-739) with the analyzers of
// the level in two kernels: the output pass (fields, mass / energy sums, the
// kinetic-energy analyzer's sum) and the enstrophy on the fields it wrote.
extern "C" int vfb_sim_output(vfb_simulation* sim, int level, double* out8, void* rho, void* vx, void* vy, void* vz,
                              void* stream)
{
    clearError();
    Level* L = levelOf(sim, level);
    if (!L)
        return VFB_ERR_INVALID_ARGUMENT;
    if (!out8)
        return setError(VFB_ERR_INVALID_ARGUMENT, "out8 is NULL");
    for (int i = 0; i < 8; ++i)
        out8[i] = 0.0;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!L->outMask.ptr) {
        // bit 0: in the fluid list; bit 1: in the kinetic-energy analyzer's set
        std::vector<uint8_t> mask(L->N, 0);
        std::vector<uint32_t> fl(L->nFluid), en(L->nEnergy);
        if ((L->nFluid && cudaMemcpyAsync(fl.data(), L->fluid.ptr, fl.size() * 4, cudaMemcpyDeviceToHost, s)) ||
            (L->nEnergy && cudaMemcpyAsync(en.data(), L->energyNodes.ptr, en.size() * 4, cudaMemcpyDeviceToHost, s)) ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return setError(VFB_ERR_CUDA, "node lists: %s", cudaGetErrorString(cudaGetLastError()));
        for (uint32_t k : fl)
            if (k < L->N)
                mask[k] |= 1u;
        for (uint32_t k : en)
            if (k < L->N)
                mask[k] |= 2u;
        if (uploadRaw(L->outMask, mask.data(), mask.size(), s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
            return setError(VFB_ERR_CUDA, "node mask upload: %s", cudaGetErrorString(cudaGetLastError()));
    }
    const bool dbl = computeIsDouble(sim->params.storage);
    const size_t bytes = L->N * (dbl ? sizeof(double) : sizeof(float));
    if (L->fieldBuffers(bytes) != cudaSuccess)
        return setError(VFB_ERR_CUDA, "field buffers: %s", cudaGetErrorString(cudaGetLastError()));
    DeviceBuffer* f = L->fields;
    const auto* geo = static_cast<const uint32_t*>(L->geo.ptr);
    const auto* nX = static_cast<const uint32_t*>(L->nX.ptr);
    const auto* nY = static_cast<const uint32_t*>(L->nY.ptr);
    const auto* nZ = static_cast<const uint32_t*>(L->nZ.ptr);
    double sums[5];
    int rc = vfb_output_pass(sim->params.storage, L->dist.ptr, L->N, geo, nX, nY, nZ,
                             static_cast<const uint8_t*>(L->outMask.ptr), L->isEven ? 1 : 0, f[0].ptr, f[1].ptr,
                             f[2].ptr, f[3].ptr, sums, stream);
    if (rc)
        return rc;
    out8[0] = sums[0];
    out8[1] = sums[1];
    out8[2] = sums[2];
    out8[3] = L->nEnergy ? sums[3] / (double)L->nEnergy : 0.0;
    out8[4] = (double)L->nEnergy;
    out8[7] = (double)L->nFluid;
    if (L->nNeg.ptr) {
        double e[2];
        rc = vfb_enstrophy(dbl ? VFB_FP64 : VFB_FP32, f[0].ptr, f[1].ptr, f[2].ptr, f[3].ptr, L->N, geo, nX, nY, nZ,
                           static_cast<const uint32_t*>(L->nNeg.ptr), e, stream);
        if (rc)
            return rc;
        out8[5] = e[0];
        out8[6] = e[1];
    }
    void* out[4] = { rho, vx, vy, vz };
    for (int i = 0; i < 4; ++i)
        if (out[i] && cudaMemcpyAsync(out[i], f[i].ptr, bytes, cudaMemcpyDeviceToHost, s) != cudaSuccess)
            return setError(VFB_ERR_CUDA, "field copy failed");
    if (cudaStreamSynchronize(s) != cudaSuccess)
        return setError(VFB_ERR_CUDA, "output: %s", cudaGetErrorString(cudaGetLastError()));
    return VFB_OK;
}

extern "C" int vfb_sim_kinetic_energy(vfb_simulation* sim, int level, double* out2, void* stream)
{
    clearError();
    Level* L = levelOf(sim, level);
    if (!L)
        return VFB_ERR_INVALID_ARGUMENT;
    if (!out2)
        return setError(VFB_ERR_INVALID_ARGUMENT, "out2 is NULL");
    out2[0] = out2[1] = 0.0;
    if (L->nEnergy == 0)
        return VFB_OK;
    double sums[3];
    const int rc = vfb_mass_and_energy(sim->params.storage, L->dist.ptr, L->N, static_cast<const uint32_t*>(L->nX.ptr),
                                       static_cast<const uint32_t*>(L->nY.ptr), static_cast<const uint32_t*>(L->nZ.ptr),
                                       static_cast<const uint32_t*>(L->energyNodes.ptr), L->nEnergy,
                                       L->isEven ? 1 : 0, sums, stream);
    if (rc)
        return rc;
    out2[0] = sums[1] / (double)L->nEnergy;
    out2[1] = (double)L->nEnergy;
    return VFB_OK;
}

extern "C" int vfb_sim_bc_epilogue_stats(vfb_simulation* sim, int level, unsigned long long* out3)
{
    clearError();
    Level* L = levelOf(sim, level);
    if (!L)
        return VFB_ERR_INVALID_ARGUMENT;
    if (!out3)
        return setError(VFB_ERR_INVALID_ARGUMENT, "out3 is NULL");
    out3[0] = out3[1] = 0;
    if (L->epilogue && L->plan)
        if (const int rc = vfb_collision_plan_epilogue_stats(L->plan, out3))
            return rc;
    unsigned long long rest = 0;
    const BcListDevice* full[4] = { &L->velocity, &L->noSlip, &L->slip, &L->geometry };
    for (int i = 0; i < 4; ++i)
        rest += L->epilogue ? L->residual[i].list.n : full[i]->n;
    out3[2] = rest;
    return VFB_OK;
}

extern "C" int vfb_sim_stress_list(vfb_simulation* sim, int level, vfb_stress_list* out)
{
    clearError();
    Level* L = levelOf(sim, level);
    if (!L)
        return VFB_ERR_INVALID_ARGUMENT;
    if (!out)
        return setError(VFB_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = stressList(L->stress, sim->params.hasWallModelMonitor != 0);
    return VFB_OK;
}

extern "C" int vfb_sim_level_state(vfb_simulation* sim, int level, void** distributions,
                                   unsigned long long* numberOfLBnodes, int* isEvenTimestep, double* omega)
{
    clearError();
    Level* L = levelOf(sim, level);
    if (!L)
        return VFB_ERR_INVALID_ARGUMENT;
    if (distributions)
        *distributions = L->dist.ptr;
    if (numberOfLBnodes)
        *numberOfLBnodes = L->N;
    if (isEvenTimestep)
        *isEvenTimestep = L->isEven ? 1 : 0;
    if (omega)
        *omega = L->omega;
    return VFB_OK;
}
