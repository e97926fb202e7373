// sim_adjoint.cu -- the adjoint of the simulation's time step: gradients of
// a flow objective with respect to the velocity-BC values and the global body
// force, by a hand-written reverse pass with checkpointing.  No counterpart in
// the reference (which has no adjoint); the step it differentiates is the
// reference's single-level UpdateGrid27 step (UpdateGrid27.cpp:54-96): K17
// collision with esoteric-twist streaming, the post-collision lists
// (velocity, no-slip, geometry) and, after the parity swap, the pressure
// lists.
//
// vfb_sim_adjoint_forward runs T steps with the adjoint's forward kernels
// (adjoint.cu: the library's operator and BC arithmetic), keeps the state
// every `interval` steps (checkpoints) and evaluates the objective
//   J = sum_j (wx_j ux + wy_j uy + wz_j uz)(node_j)
// on the final state.  vfb_sim_adjoint_backward seeds lam = dJ/df on the
// final state, then walks the checkpoint segments backwards: it restores a
// checkpoint into a work array, recomputes the segment's steps while taping
// each step's collision inputs and BC inputs, and applies the adjoint steps
// in reverse order (pressure, geometry, no-slip, velocity, collision).  The
// BC adjoints accumulate dJ/dU per velocity-list entry; the collision adjoint
// gives dJ/d(half force), which is dJ/dg times 1/2 * forceFactor.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
#include <unordered_map>
#include <utility>
#include <vector>

#include "adjoint.cuh"
#include "capi_common.cuh"
#include "sim_state.hpp"

namespace vfb
{
struct AdjointState {
    int storage = -1;
    unsigned steps = 0, interval = 0;
    std::vector<DeviceBuffer*> checkpoints;
    std::vector<char> checkpointEven;
    DeviceBuffer finalState, work, lam;
    bool finalEven = true;
    bool ready = false;
    // per segment: the collision tape and the BC records of every step
    DeviceBuffer tape, recVelocity, recNoSlip, recGeometry, recPressure;
    DeviceBuffer tmpVelocity, tmpNoSlip, tmpGeometry, tmpPressure;
    std::vector<size_t> pressureOffset; // first entry of each pressure list in recPressure / tmpPressure
    size_t pressureTotal = 0;
    DeviceBuffer objNodes, objW[3], partials, accForce, gVelocity;
    DeviceBuffer forcePartials; // 3 per collision block, accumulated over a backward pass
    DeviceBuffer fluidLocations; // 8 * nFluid: the fluid list's node locations (vfb_bc_locations)
    uint32_t nObj = 0;
    int velocityKind = -1, noSlipKind = -1, geometryKind = -1;
    bool pressure = false;
    // the post-collision lists write cells no other list reads or writes, so
    // each step launches them together (-1: not checked yet)
    int listsCommute = -1;
    // the forward pass recorded the tapes and BC records of its only segment:
    // the backward pass reverses them without recomputing the steps
    bool taped = false;
    // captured backward segments (recompute with tapes, then the reverse
    // steps), keyed by the segment length and the parity it starts from
    cudaStream_t captureStream = nullptr;
    std::map<std::pair<unsigned, int>, cudaGraphExec_t> segments;
    void dropGraphs()
    {
        for (auto& g : segments)
            cudaGraphExecDestroy(g.second);
        segments.clear();
    }
    ~AdjointState()
    {
        dropGraphs();
        if (captureStream)
            cudaStreamDestroy(captureStream);
        for (auto* c : checkpoints)
            delete c;
    }
};

void destroyAdjoint(AdjointState* a) { delete a; }

namespace
{
cudaError_t ensure(DeviceBuffer& b, size_t bytes)
{
    if (b.ptr && b.bytes >= bytes)
        return cudaSuccess;
    if (b.ptr) {
        cudaFree(b.ptr);
        b.ptr = nullptr;
    }
    return b.allocate(bytes);
}

template <class T>
T* as(DeviceBuffer& b)
{
    return static_cast<T*>(b.ptr);
}

// the supported configuration: one level, K17, FP32 or FP64, interpolated
// velocity / no-slip lists, non-equilibrium pressure lists, no slip list
int checkSupported(const vfb_simulation& S)
{
    const vfb_sim_params& P = S.params;
    if (S.levels.size() != 1)
        return setError(VFB_ERR_UNSUPPORTED, "the adjoint covers single-level simulations (this one has %zu levels)",
                        S.levels.size());
    if (P.collisionKernel != 0)
        return setError(VFB_ERR_UNSUPPORTED, "the adjoint covers the K17 collision");
    if (P.storage != VFB_FP32 && P.storage != VFB_FP64)
        return setError(VFB_ERR_UNSUPPORTED, "the adjoint needs FP32 or FP64 storage");
    const Level& L = *S.levels[0];
    if (L.velocity.n && P.velocityBC != VFB_BC_VELOCITY_INTERPOLATED)
        return setError(VFB_ERR_UNSUPPORTED, "the adjoint covers VelocityInterpolatedCompressible on the velocity list");
    if (L.noSlip.n && P.noSlipBC >= 0 && P.noSlipBC != VFB_BC_NOSLIP_INTERPOLATED)
        return setError(VFB_ERR_UNSUPPORTED, "the adjoint covers NoSlipInterpolatedCompressible on the no-slip list");
    if (L.geometry.n && P.geometryBC >= 0 && P.geometryBC != VFB_BC_NOSLIP_INTERPOLATED)
        return setError(VFB_ERR_UNSUPPORTED, "the adjoint covers NoSlipInterpolatedCompressible on the geometry list");
    if (L.slip.n && P.slipBC >= 0)
        return setError(VFB_ERR_UNSUPPORTED, "the adjoint does not cover the slip list");
    if (L.stress.n && P.stressBC >= 0)
        return setError(VFB_ERR_UNSUPPORTED, "the adjoint does not cover the stress (wall-model) list");
    size_t np = 0;
    for (const auto* p : L.pressure)
        np += p->n;
    if (np && P.pressureBC > 0)
        return setError(VFB_ERR_UNSUPPORTED, "the adjoint covers PressureNonEquilibriumCompressible pressure lists");
    return VFB_OK;
}

int cudaFail(const char* what)
{
    return setError(VFB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(cudaGetLastError()));
}

template <class R>
struct Stepper {
    vfb_simulation& S;
    Level& L;
    AdjointState& A;
    cudaStream_t s;
    K17Rates<R> rates;
    R fx, fy, fz;
    BcLattice<R> lat;

    Stepper(vfb_simulation& sim, AdjointState& a, cudaStream_t stream)
        : S(sim), L(*sim.levels[0]), A(a), s(stream)
    {
        const vfb_sim_params& P = S.params;
        // the forward collision's per-launch constants (collision.cu)
        rates = makeK17Rates<R>((R)L.omega, (R)P.quadricLimiters[0], (R)P.quadricLimiters[1], (R)P.quadricLimiters[2]);
        const R factor = (R)L.forceFactor;
        fx = (R)P.forces[0] * R(0.5) * factor;
        fy = (R)P.forces[1] * R(0.5) * factor;
        fz = (R)P.forces[2] * R(0.5) * factor;
        lat = BcLattice<R>{ L.N, as<const uint32_t>(L.nX), as<const uint32_t>(L.nY), as<const uint32_t>(L.nZ),
                            (R)L.omega };
    }

    const uint32_t* nX() { return as<const uint32_t>(L.nX); }
    const uint32_t* nY() { return as<const uint32_t>(L.nY); }
    const uint32_t* nZ() { return as<const uint32_t>(L.nZ); }

    R* slotOf(DeviceBuffer& b, int slot, size_t n) { return slot < 0 ? nullptr : as<R>(b) + (size_t)slot * 27 * n; }

    adjoint::PostList<R> postList(BcListDevice& B, int kind, R* rec, R* tmp, double* gV)
    {
        return adjoint::PostList<R>{ kind, as<const int32_t>(B.k), as<const uint32_t>(B.locations), as<const R>(B.q),
                                     B.n, as<const R>(B.vx), as<const R>(B.vy), as<const R>(B.vz), rec, tmp, gV };
    }

    // one step of the forward schedule on `dist` (parity `even` flips); with
    // slot >= 0 the step's inputs are recorded in that slot of the tapes
    int forward(R* dist, bool& even, int slot)
    {
        if (const int rc = adjoint::collision<R>(dist, L.N, nX(), nY(), nZ(), as<const uint32_t>(L.fluid),
                                                 as<const uint32_t>(A.fluidLocations), L.nFluid, rates, fx, fy, fz,
                                                 even, slotOf(A.tape, slot, L.nFluid), s))
            return rc;
        BcLattice<R> t = lat;
        struct Item {
            BcListDevice* list;
            int kind;
            DeviceBuffer* rec;
        } items[3] = { { &L.velocity, A.velocityKind, &A.recVelocity },
                       { &L.noSlip, A.noSlipKind, &A.recNoSlip },
                       { &L.geometry, A.geometryKind, &A.recGeometry } };
        if (A.listsCommute == 1) {
            adjoint::PostLists<R> P;
            for (Item& it : items)
                if (it.list->n && it.kind >= 0)
                    P.list[P.count++] = postList(*it.list, it.kind, slotOf(*it.rec, slot, it.list->n), nullptr,
                                                 nullptr);
            if (const int rc = adjoint::postBCLists<R>(dist, t, P, even, s))
                return rc;
        }
        for (Item& it : items) {
            if (A.listsCommute == 1 || it.list->n == 0 || it.kind < 0)
                continue;
            if (const int rc = adjoint::postBC<R>(it.kind, dist, t, as<const int32_t>(it.list->k),
                                                  as<const uint32_t>(it.list->locations), as<const R>(it.list->q),
                                                  it.list->n, as<const R>(it.list->vx),
                                                  as<const R>(it.list->vy), as<const R>(it.list->vz), even,
                                                  slotOf(*it.rec, slot, it.list->n), s))
                return rc;
        }
        even = !even;
        if (A.pressure)
            for (size_t p = 0; p < L.pressure.size(); ++p) {
                PressureListDevice& P = *L.pressure[p];
                if (P.n == 0)
                    continue;
                R* rec = slot < 0 ? nullptr : as<R>(A.recPressure) + (size_t)slot * 27 * A.pressureTotal +
                                                  27 * A.pressureOffset[p];
                if (const int rc = adjoint::pressureBC<R>(dist, t, as<const int32_t>(P.k), as<const int32_t>(P.kN),
                                                          as<const R>(P.rho), P.n, P.direction, even, rec, s))
                    return rc;
            }
        return VFB_OK;
    }

    // the adjoint of the step recorded in `slot`, whose collision ran with parity `even`
    int reverse(bool even, int slot)
    {
        R* lam = as<R>(A.lam);
        if (A.pressure)
            for (size_t p = L.pressure.size(); p-- > 0;) {
                PressureListDevice& P = *L.pressure[p];
                if (P.n == 0)
                    continue;
                const size_t off = 27 * A.pressureOffset[p];
                const R* rec = as<R>(A.recPressure) + (size_t)slot * 27 * A.pressureTotal + off;
                if (const int rc = adjoint::pressureBCAdjoint<R>(lam, lat, as<const int32_t>(P.k),
                                                                 as<const int32_t>(P.kN), as<const R>(P.rho), P.n,
                                                                 P.direction, !even, rec, as<R>(A.tmpPressure) + off,
                                                                 s))
                    return rc;
            }
        struct Item {
            BcListDevice* list;
            int kind;
            DeviceBuffer* rec;
            DeviceBuffer* tmp;
            double* gV;
        } items[3] = { { &L.geometry, A.geometryKind, &A.recGeometry, &A.tmpGeometry, nullptr },
                       { &L.noSlip, A.noSlipKind, &A.recNoSlip, &A.tmpNoSlip, nullptr },
                       { &L.velocity, A.velocityKind, &A.recVelocity, &A.tmpVelocity, as<double>(A.gVelocity) } };
        if (A.listsCommute == 1) {
            adjoint::PostLists<R> P;
            for (Item& it : items)
                if (it.list->n && it.kind >= 0)
                    P.list[P.count++] = postList(*it.list, it.kind, slotOf(*it.rec, slot, it.list->n), as<R>(*it.tmp),
                                                 it.gV);
            if (const int rc = adjoint::postBCAdjointLists<R>(lam, lat, P, even, s))
                return rc;
        }
        for (Item& it : items) {
            if (A.listsCommute == 1 || it.list->n == 0 || it.kind < 0)
                continue;
            if (const int rc = adjoint::postBCAdjoint<R>(
                    it.kind, lam, lat, as<const int32_t>(it.list->k), as<const uint32_t>(it.list->locations),
                    as<const R>(it.list->q), it.list->n,
                    as<const R>(it.list->vx), as<const R>(it.list->vy), as<const R>(it.list->vz), even,
                    slotOf(*it.rec, slot, it.list->n), as<R>(*it.tmp), it.gV, s))
                return rc;
        }
        return adjoint::collisionAdjoint<R>(lam, L.N, nX(), nY(), nZ(), as<const uint32_t>(L.fluid),
                                            as<const uint32_t>(A.fluidLocations), L.nFluid, rates, fx, fy, fz, even,
                                            slotOf(A.tape, slot, L.nFluid), as<double>(A.forcePartials), s);
    }
};

template <class R>
int objectiveValue(vfb_simulation& S, AdjointState& A, const R* dist, bool even, double* J, R* lam, double seed,
                   cudaStream_t s)
{
    Level& L = *S.levels[0];
    const unsigned blocks = adjoint::objectiveBlocks(A.nObj);
    if (cudaMemsetAsync(A.accForce.ptr, 0, 4 * sizeof(double), s) != cudaSuccess)
        return cudaFail("objective accumulator");
    if (const int rc = adjoint::objective<R>(dist, L.N, as<const uint32_t>(L.nX), as<const uint32_t>(L.nY),
                                             as<const uint32_t>(L.nZ), as<const uint32_t>(A.objNodes),
                                             as<const double>(A.objW[0]), as<const double>(A.objW[1]),
                                             as<const double>(A.objW[2]), A.nObj, even, as<double>(A.partials), lam,
                                             seed, s))
        return rc;
    if (const int rc = adjoint::reducePartials(as<double>(A.partials), blocks, 1, as<double>(A.accForce) + 3, 1.0, s))
        return rc;
    if (J) {
        if (cudaMemcpyAsync(J, as<double>(A.accForce) + 3, sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return cudaFail("objective copy");
    }
    return VFB_OK;
}

// Whether the post-collision lists of the adjoint (velocity, no-slip,
// geometry) can run in one launch per step: in both parities, no cell a list
// writes (the cell of inv(d) in the other view, for each link d with
// 0 <= q_d <= 1) is written by another list or is one of the 27 cells
// another list's nodes read.  Then the lists commute, forward and adjoint.
// VFB_ADJOINT_SEPARATE_LISTS=1 keeps one launch per list (for comparisons).
template <class R>
int listsCommute(vfb_simulation& S, AdjointState& A, cudaStream_t s, bool& result)
{
    result = false;
    if (const char* env = std::getenv("VFB_ADJOINT_SEPARATE_LISTS"))
        if (env[0] == '1')
            return VFB_OK;
    Level& L = *S.levels[0];
    struct Item {
        BcListDevice* list;
        int kind;
    } items[3] = { { &L.velocity, A.velocityKind }, { &L.noSlip, A.noSlipKind }, { &L.geometry, A.geometryKind } };
    std::vector<std::vector<uint32_t>> locs;
    std::vector<std::vector<R>> qs;
    for (Item& it : items) {
        if (it.list->n == 0 || it.kind < 0)
            continue;
        const uint32_t n = it.list->n;
        locs.emplace_back(8ull * n);
        qs.emplace_back(27ull * n);
        if (!it.list->locations.ptr ||
            cudaMemcpyAsync(locs.back().data(), it.list->locations.ptr, 8ull * n * sizeof(uint32_t),
                            cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaMemcpyAsync(qs.back().data(), it.list->q.ptr, 27ull * n * sizeof(R), cudaMemcpyDeviceToHost, s) !=
                cudaSuccess)
            return cudaFail("BC list download");
    }
    if (cudaStreamSynchronize(s) != cudaSuccess)
        return cudaFail("BC list download");
    if (locs.size() < 2)
        return VFB_OK; // nothing to launch together
    const unsigned long long N = L.N;
    for (int parity = 0; parity < 2; ++parity) {
        const bool even = parity == 0;
        std::unordered_map<unsigned long long, int> written; // cell -> list
        for (size_t l = 0; l < locs.size(); ++l) {
            const size_t n = locs[l].size() / 8;
            for (size_t i = 0; i < n; ++i)
                for (int d = 1; d < 27; ++d) {
                    const R q = qs[l][(size_t)d * n + i];
                    if (!(q >= R(0) && q <= R(1)))
                        continue;
                    const int e = inv(d);
                    const unsigned long long c =
                        (unsigned long long)(even ? slot<false>(e) : slot<true>(e)) * N + locs[l][(size_t)loc(e) * n + i];
                    const auto ins = written.emplace(c, (int)l);
                    if (!ins.second && ins.first->second != (int)l)
                        return VFB_OK; // two lists write one cell
                }
        }
        for (size_t l = 0; l < locs.size(); ++l) {
            const size_t n = locs[l].size() / 8;
            for (size_t i = 0; i < n; ++i)
                for (int d = 0; d < 27; ++d) {
                    const int r = inv(d);
                    const unsigned long long c =
                        (unsigned long long)(even ? slot<true>(r) : slot<false>(r)) * N + locs[l][(size_t)loc(r) * n + i];
                    const auto it = written.find(c);
                    if (it != written.end() && it->second != (int)l)
                        return VFB_OK; // a list reads a cell another list writes
                }
        }
    }
    result = true;
    return VFB_OK;
}

// the buffers of one backward segment (tapes, records, scratch); a
// reallocation drops the captured segment graphs, which hold their addresses
template <class R>
int ensureSegmentBuffers(vfb_simulation& S, AdjointState& A)
{
    Level& L = *S.levels[0];
    const size_t stateBytes = 27ull * L.N * sizeof(R);
    const unsigned I = A.interval;
    auto perStep = [&](DeviceBuffer& b, size_t n) { return ensure(b, std::max<size_t>(1, (size_t)I * 27 * n * sizeof(R))); };
    auto once = [&](DeviceBuffer& b, size_t n) { return ensure(b, std::max<size_t>(1, 27 * n * sizeof(R))); };
    DeviceBuffer* held[] = { &A.work, &A.lam, &A.tape, &A.recVelocity, &A.recNoSlip, &A.recGeometry, &A.recPressure,
                             &A.tmpVelocity, &A.tmpNoSlip, &A.tmpGeometry, &A.tmpPressure, &A.gVelocity,
                             &A.partials, &A.accForce, &A.forcePartials };
    std::vector<void*> before;
    for (DeviceBuffer* b : held)
        before.push_back(b->ptr);
    if (ensure(A.work, stateBytes) || ensure(A.lam, stateBytes) || perStep(A.tape, L.nFluid) ||
        perStep(A.recVelocity, L.velocity.n) || perStep(A.recNoSlip, L.noSlip.n) ||
        perStep(A.recGeometry, L.geometry.n) || perStep(A.recPressure, A.pressureTotal) ||
        once(A.tmpVelocity, L.velocity.n) || once(A.tmpNoSlip, L.noSlip.n) || once(A.tmpGeometry, L.geometry.n) ||
        once(A.tmpPressure, A.pressureTotal) ||
        ensure(A.gVelocity, std::max<size_t>(1, 3ull * L.velocity.n * sizeof(double))) ||
        ensure(A.forcePartials, 3ull * std::max(1u, adjoint::collisionBlocks(L.nFluid)) * sizeof(double)))
        return cudaFail("adjoint buffers");
    for (size_t i = 0; i < before.size(); ++i)
        if (held[i]->ptr != before[i]) {
            A.dropGraphs();
            break;
        }
    return VFB_OK;
}

template <class R>
int adjointForward(vfb_simulation& S, AdjointState& A, unsigned steps, double* J, cudaStream_t s)
{
    Level& L = *S.levels[0];
    const size_t stateBytes = 27ull * L.N * sizeof(R);
    const unsigned segments = (steps + A.interval - 1) / A.interval;
    while (A.checkpoints.size() < segments)
        A.checkpoints.push_back(new DeviceBuffer);
    A.checkpointEven.assign(segments, 1);
    for (unsigned c = 0; c < segments; ++c)
        if (ensure(*A.checkpoints[c], stateBytes) != cudaSuccess)
            return cudaFail("checkpoint allocation");
    // the fluid list's location table, once (the collision kernels of both
    // passes read it instead of walking the neighbour arrays)
    if (!A.fluidLocations.ptr && L.nFluid) {
        if (ensure(A.fluidLocations, 8ull * L.nFluid * sizeof(uint32_t)) != cudaSuccess)
            return cudaFail("fluid location table");
        if (const int rc = vfb_bc_locations(as<const int32_t>(L.fluid), L.nFluid, as<const uint32_t>(L.nX),
                                            as<const uint32_t>(L.nY), as<const uint32_t>(L.nZ),
                                            as<uint32_t>(A.fluidLocations), s))
            return rc;
    }
    if (A.listsCommute < 0) {
        bool ok = false;
        if (const int rc = listsCommute<R>(S, A, s, ok))
            return rc;
        A.listsCommute = ok ? 1 : 0;
    }
    // one segment: the forward pass records its tapes itself (the memory the
    // backward pass would take for them anyway), and nothing is recomputed
    A.taped = segments == 1;
    if (A.taped)
        if (const int rc = ensureSegmentBuffers<R>(S, A))
            return rc;
    Stepper<R> st(S, A, s);
    R* dist = as<R>(L.dist);
    bool even = L.isEven;
    for (unsigned t = 0; t < steps; ++t) {
        if (t % A.interval == 0) {
            const unsigned c = t / A.interval;
            if (cudaMemcpyAsync(A.checkpoints[c]->ptr, dist, stateBytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
                return cudaFail("checkpoint copy");
            A.checkpointEven[c] = even ? 1 : 0;
        }
        if (const int rc = st.forward(dist, even, A.taped ? (int)t : -1))
            return rc;
    }
    L.isEven = even;
    S.stepsRun += steps;
    if (ensure(A.finalState, stateBytes) != cudaSuccess ||
        cudaMemcpyAsync(A.finalState.ptr, dist, stateBytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
        return cudaFail("final state copy");
    A.finalEven = even;
    return objectiveValue<R>(S, A, dist, even, J, nullptr, 0.0, s);
}

template <class R>
int adjointBackward(vfb_simulation& S, AdjointState& A, double seed, double* dVelocity, double* dForces,
                    cudaStream_t s)
{
    Level& L = *S.levels[0];
    const size_t stateBytes = 27ull * L.N * sizeof(R);
    const unsigned I = A.interval;
    if (const int rc = ensureSegmentBuffers<R>(S, A))
        return rc;
    if (cudaMemsetAsync(A.lam.ptr, 0, stateBytes, s) != cudaSuccess ||
        cudaMemsetAsync(A.gVelocity.ptr, 0, A.gVelocity.bytes, s) != cudaSuccess)
        return cudaFail("adjoint clear");
    // seed: lam = seed * dJ/df on the final state
    if (const int rc = objectiveValue<R>(S, A, as<const R>(A.finalState), A.finalEven, nullptr, as<R>(A.lam), seed, s))
        return rc;
    if (cudaMemsetAsync(A.accForce.ptr, 0, 3 * sizeof(double), s) != cudaSuccess ||
        cudaMemsetAsync(A.forcePartials.ptr, 0, A.forcePartials.bytes, s) != cudaSuccess)
        return cudaFail("force accumulator");
    if (!A.captureStream && cudaStreamCreateWithFlags(&A.captureStream, cudaStreamNonBlocking) != cudaSuccess)
        return cudaFail("capture stream");
    // one segment: recompute its steps from the work array with tapes (unless
    // the forward pass taped them), then the adjoint steps in reverse order
    auto segment = [&](Stepper<R>& st, unsigned len, bool even) -> int {
        std::vector<char> evenAt(len);
        for (unsigned j = 0; j < len; ++j) {
            evenAt[j] = even ? 1 : 0;
            if (A.taped)
                even = !even; // the parity flips once per step
            else if (const int rc = st.forward(as<R>(A.work), even, (int)j))
                return rc;
        }
        for (unsigned j = len; j-- > 0;)
            if (const int rc = st.reverse(evenAt[j] != 0, (int)j))
                return rc;
        return VFB_OK;
    };
    const unsigned segments = (A.steps + I - 1) / I;
    for (unsigned c = segments; c-- > 0;) {
        const unsigned t0 = c * I;
        const unsigned len = std::min(I, A.steps - t0);
        if (!A.taped &&
            cudaMemcpyAsync(A.work.ptr, A.checkpoints[c]->ptr, stateBytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
            return cudaFail("checkpoint restore");
        const bool even = A.checkpointEven[c] != 0;
        const auto key = std::make_pair(len, (even ? 1 : 0) | (A.taped ? 2 : 0));
        auto it = A.segments.find(key);
        if (it == A.segments.end()) {
            // capture the segment's launches once; every segment of this length
            // and starting parity replays the same graph (same buffers)
            Stepper<R> cst(S, A, A.captureStream);
            if (cudaStreamBeginCapture(A.captureStream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
                return cudaFail("begin capture");
            const int rc = segment(cst, len, even);
            cudaGraph_t graph = nullptr;
            const cudaError_t e = cudaStreamEndCapture(A.captureStream, &graph);
            if (rc != VFB_OK) {
                if (graph)
                    cudaGraphDestroy(graph);
                return rc;
            }
            cudaGraphExec_t exec = nullptr;
            const cudaError_t ie = e == cudaSuccess && graph ? cudaGraphInstantiate(&exec, graph, 0) : e;
            if (graph)
                cudaGraphDestroy(graph);
            if (ie != cudaSuccess)
                return setError(VFB_ERR_CUDA, "segment graph: %s", cudaGetErrorString(ie));
            it = A.segments.emplace(key, exec).first;
        }
        if (cudaGraphLaunch(it->second, s) != cudaSuccess)
            return cudaFail("segment graph launch");
    }
    // the force adjoint: every block's sum over all steps, reduced once in block order
    if (const int rc = adjoint::reducePartials(as<double>(A.forcePartials), adjoint::collisionBlocks(L.nFluid), 3,
                                               as<double>(A.accForce), 0.5 * L.forceFactor, s))
        return rc;
    if (dVelocity && L.velocity.n &&
        cudaMemcpyAsync(dVelocity, A.gVelocity.ptr, 3ull * L.velocity.n * sizeof(double), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess)
        return cudaFail("velocity gradient copy");
    double g[3] = { 0, 0, 0 };
    if (cudaMemcpyAsync(g, A.accForce.ptr, sizeof(g), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return cudaFail("backward pass");
    if (dForces)
        for (int c = 0; c < 3; ++c)
            dForces[c] = g[c];
    return VFB_OK;
}
} // namespace
} // namespace vfb

using namespace vfb;

extern "C" int vfb_sim_set_forces(vfb_simulation* sim, const double* forces)
{
    clearError();
    if (!sim || !forces)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    for (int c = 0; c < 3; ++c)
        sim->params.forces[c] = forces[c];
    // captured graphs hold the old force in their kernel arguments
    for (auto& g : sim->graphs)
        cudaGraphExecDestroy(g.second);
    sim->graphs.clear();
    if (sim->adjoint) {
        sim->adjoint->ready = false;
        sim->adjoint->dropGraphs();
    }
    return VFB_OK;
}

extern "C" int vfb_sim_set_velocity_bc(vfb_simulation* sim, int level, const double* vx, const double* vy,
                                       const double* vz, void* stream)
{
    clearError();
    if (!sim || level < 0 || level >= (int)sim->levels.size())
        return setError(VFB_ERR_INVALID_ARGUMENT, "no level %d", level);
    if (!vx || !vy || !vz)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL velocity array");
    BcListDevice& B = sim->levels[level]->velocity;
    if (B.n == 0)
        return VFB_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const bool dbl = sim->params.storage == VFB_FP64;
    const double* src[3] = { vx, vy, vz };
    DeviceBuffer* dst[3] = { &B.vx, &B.vy, &B.vz };
    std::vector<float> f(B.n);
    for (int c = 0; c < 3; ++c) {
        if (!dst[c]->ptr)
            return setError(VFB_ERR_CONFIGURATION, "the velocity list has no velocity arrays");
        cudaError_t e;
        if (dbl) {
            e = cudaMemcpyAsync(dst[c]->ptr, src[c], B.n * sizeof(double), cudaMemcpyHostToDevice, s);
        } else {
            for (uint32_t i = 0; i < B.n; ++i)
                f[i] = (float)src[c][i];
            e = cudaMemcpyAsync(dst[c]->ptr, f.data(), B.n * sizeof(float), cudaMemcpyHostToDevice, s);
        }
        if (e != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
            return cudaFail("velocity upload");
    }
    // the entries of the velocity list the BC epilogue leaves to the separate launch
    Level& L = *sim->levels[level];
    if (L.epilogue && L.residual[0].list.n) {
        ResidualList& R = L.residual[0];
        DeviceBuffer* rdst[3] = { &R.list.vx, &R.list.vy, &R.list.vz };
        std::vector<double> g(R.index.size());
        std::vector<float> gf(R.index.size());
        for (int c = 0; c < 3; ++c) {
            for (size_t j = 0; j < R.index.size(); ++j) {
                g[j] = src[c][R.index[j]];
                gf[j] = (float)g[j];
            }
            const cudaError_t e = dbl ? cudaMemcpyAsync(rdst[c]->ptr, g.data(), g.size() * sizeof(double),
                                                        cudaMemcpyHostToDevice, s)
                                      : cudaMemcpyAsync(rdst[c]->ptr, gf.data(), gf.size() * sizeof(float),
                                                        cudaMemcpyHostToDevice, s);
            if (e != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
                return cudaFail("velocity upload");
        }
    }
    if (sim->adjoint)
        sim->adjoint->ready = false;
    return VFB_OK;
}

extern "C" int vfb_sim_adjoint_forward(vfb_simulation* sim, unsigned int steps, unsigned int checkpointInterval,
                                       const uint32_t* objectiveNodes, const double* wx, const double* wy,
                                       const double* wz, uint32_t numberOfObjectiveNodes, double* J, void* stream)
{
    clearError();
    if (!sim || !J)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    if (checkpointInterval == 0)
        return setError(VFB_ERR_INVALID_ARGUMENT, "checkpoint interval must be positive");
    if (numberOfObjectiveNodes && (!objectiveNodes || !wx || !wy || !wz))
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL objective array");
    if (const int rc = checkSupported(*sim))
        return rc;
    Level& L = *sim->levels[0];
    for (uint32_t j = 0; j < numberOfObjectiveNodes; ++j)
        if (objectiveNodes[j] == 0 || objectiveNodes[j] >= L.N)
            return setError(VFB_ERR_OUT_OF_RANGE, "objective node %u outside 1..%llu", objectiveNodes[j], L.N - 1);
    if (!sim->adjoint)
        sim->adjoint = new AdjointState;
    AdjointState& A = *sim->adjoint;
    if (A.interval != checkpointInterval)
        A.dropGraphs(); // the segment graphs are sized by the interval
    A.storage = sim->params.storage;
    A.steps = steps;
    A.interval = checkpointInterval;
    A.ready = false;
    const vfb_sim_params& P = sim->params;
    A.velocityKind = L.velocity.n ? VFB_BC_VELOCITY_INTERPOLATED : -1;
    A.noSlipKind = L.noSlip.n && P.noSlipBC >= 0 ? VFB_BC_NOSLIP_INTERPOLATED : -1;
    A.geometryKind = L.geometry.n && P.geometryBC >= 0 ? VFB_BC_NOSLIP_INTERPOLATED : -1;
    A.pressure = P.pressureBC == 0;
    A.pressureOffset.clear();
    A.pressureTotal = 0;
    for (const auto* p : L.pressure) {
        A.pressureOffset.push_back(A.pressureTotal);
        A.pressureTotal += p->n;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    A.nObj = numberOfObjectiveNodes;
    const size_t n = std::max<uint32_t>(1, numberOfObjectiveNodes);
    const unsigned partials = std::max(adjoint::collisionBlocks(L.nFluid), adjoint::objectiveBlocks(A.nObj));
    if (ensure(A.objNodes, n * sizeof(uint32_t)) || ensure(A.objW[0], n * sizeof(double)) ||
        ensure(A.objW[1], n * sizeof(double)) || ensure(A.objW[2], n * sizeof(double)) ||
        ensure(A.partials, 3ull * std::max(1u, partials) * sizeof(double)) || ensure(A.accForce, 4 * sizeof(double)))
        return cudaFail("objective buffers");
    if (numberOfObjectiveNodes) {
        const double* w[3] = { wx, wy, wz };
        if (cudaMemcpyAsync(A.objNodes.ptr, objectiveNodes, numberOfObjectiveNodes * sizeof(uint32_t),
                            cudaMemcpyHostToDevice, s) != cudaSuccess)
            return cudaFail("objective upload");
        for (int c = 0; c < 3; ++c)
            if (cudaMemcpyAsync(A.objW[c].ptr, w[c], numberOfObjectiveNodes * sizeof(double), cudaMemcpyHostToDevice,
                                s) != cudaSuccess)
                return cudaFail("objective upload");
    }
    const int rc = sim->params.storage == VFB_FP64 ? adjointForward<double>(*sim, A, steps, J, s)
                                                   : adjointForward<float>(*sim, A, steps, J, s);
    if (rc == VFB_OK && numberOfObjectiveNodes == 0)
        *J = 0.0;
    A.ready = rc == VFB_OK;
    return rc;
}

extern "C" int vfb_sim_adjoint_backward(vfb_simulation* sim, double seed, double* dVelocity, double* dForces,
                                        void* stream)
{
    clearError();
    if (!sim)
        return setError(VFB_ERR_INVALID_ARGUMENT, "sim is NULL");
    if (!sim->adjoint || !sim->adjoint->ready)
        return setError(VFB_ERR_CONFIGURATION, "no adjoint forward pass to differentiate (run vfb_sim_adjoint_forward "
                                               "after the last change of forces or BC velocities)");
    AdjointState& A = *sim->adjoint;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    return A.storage == VFB_FP64 ? adjointBackward<double>(*sim, A, seed, dVelocity, dForces, s)
                                 : adjointBackward<float>(*sim, A, seed, dVelocity, dForces, s);
}

extern "C" int vfb_sim_adjoint_schedule(const vfb_simulation* sim, int* out2)
{
    clearError();
    if (!sim || !out2)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!sim->adjoint || !sim->adjoint->ready)
        return setError(VFB_ERR_CONFIGURATION, "no adjoint forward pass");
    out2[0] = sim->adjoint->listsCommute == 1 ? 1 : 0;
    out2[1] = sim->adjoint->taped ? 1 : 0;
    return VFB_OK;
}
