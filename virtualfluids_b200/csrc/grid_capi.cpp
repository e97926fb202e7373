// grid_capi.cpp -- C ABI of the grid builder: build a multi-level sparse grid
// from a flat description and export the arrays the GPU solver consumes.
#include <cmath>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "capi_common.cuh"
#include "d3q27.cuh"
#include "grid_builder.hpp"

namespace
{
// a primitive from 7 spec values: kind (1 cuboid, 2 sphere, 3 cylinder,
// 4 vertical cylinder) and its parameters
vfb::grid::Solid primitiveFrom(const double* p)
{
    using vfb::grid::Box;
    using vfb::grid::Solid;
    Solid solid;
    if (p[0] == 3 || p[0] == 4) {
        // 4: VerticalCylinder (VerticalCylinder.cpp:97-112), the same test about the z axis
        solid.kind = Solid::Kind::Cylinder;
        solid.cx = p[1];
        solid.cy = p[2];
        solid.cz = p[3];
        solid.r = p[4];
        solid.height = p[5];
        solid.axis = p[0] == 4 ? 2 : (int)p[6];
        if (solid.axis < 0 || solid.axis > 2)
            throw std::invalid_argument("cylinder axis must be 0, 1 or 2");
    } else if (p[0] == 2) {
        solid.kind = Solid::Kind::Sphere;
        solid.cx = p[1];
        solid.cy = p[2];
        solid.cz = p[3];
        solid.r = p[4];
    } else {
        solid.box = Box { p[1], p[2], p[3], p[4], p[5], p[6] };
    }
    return solid;
}

using namespace vfb::grid;

struct Exported {
    std::map<std::string, std::vector<char>> data;
    std::map<std::string, int> elem;
    template <class T>
    void put(const std::string& name, const std::vector<T>& v)
    {
        std::vector<char>& d = data[name];
        d.resize(v.size() * sizeof(T));
        if (!v.empty())
            std::memcpy(d.data(), v.data(), d.size());
        elem[name] = (int)sizeof(T);
    }
};

struct GridHandle {
    GridBuilder builder;
    std::vector<Exported> levels;
};

SideType sideOf(int s)
{
    if (s < 0 || s > 5)
        throw std::invalid_argument("side id must be 0..5");
    return (SideType)s;
}

// the stress parameters of side slot i: spec[176 + 3 i .. 178 + 3 i]
constexpr int kStressBase = 176;
constexpr int kSpecWithStress = kStressBase + 18;

void applyBC(GridBuilder& b, int side, int type, double v0, double v1, double v2, const double* stress)
{
    switch (type) {
    case 0: break;
    case 1: b.setNoSlipBoundaryCondition(sideOf(side)); break;
    case 2: b.setVelocityBoundaryCondition(sideOf(side), v0, v1, v2); break;
    case 3: b.setPressureBoundaryCondition(sideOf(side), v0); break;
    case 4: b.setSlipBoundaryCondition(sideOf(side), v0, v1, v2); break;
    case 5:
        if (!stress)
            throw std::invalid_argument("a stress BC needs the spec's stress block (194 values)");
        if (!(stress[0] >= 0) || stress[0] != std::floor(stress[0]))
            throw std::invalid_argument("the stress BC's sampling offset must be a whole number >= 0");
        b.setStressBoundaryCondition(sideOf(side), v0, v1, v2, (uint32_t)stress[0], stress[1], stress[2]);
        break;
    default: throw std::invalid_argument("unknown boundary-condition type");
    }
}

void concatenate(const std::vector<BCList>& lists, Exported& E, const std::string& prefix, bool velocity, bool slip)
{
    std::vector<int32_t> k;
    std::vector<double> vx, vy, vz, nx, ny, nz;
    size_t n = 0;
    for (const auto& l : lists)
        n += l.size();
    std::vector<double> q(27 * n, -1.0);
    size_t at = 0;
    for (const auto& l : lists) {
        const size_t m = l.size();
        for (size_t i = 0; i < m; ++i) {
            k.push_back(l.k[i]);
            if (velocity) {
                vx.push_back(l.vx[i]);
                vy.push_back(l.vy[i]);
                vz.push_back(l.vz[i]);
            }
            if (slip) {
                nx.push_back(l.normalX[i]);
                ny.push_back(l.normalY[i]);
                nz.push_back(l.normalZ[i]);
            }
            for (int d = 0; d < 27; ++d)
                q[(size_t)d * n + at + i] = l.q[(size_t)d * m + i];
        }
        at += m;
    }
    E.put(prefix + ".k", k);
    E.put(prefix + ".q", q);
    if (velocity) {
        E.put(prefix + ".vx", vx);
        E.put(prefix + ".vy", vy);
        E.put(prefix + ".vz", vz);
    }
    if (slip) {
        E.put(prefix + ".nx", nx);
        E.put(prefix + ".ny", ny);
        E.put(prefix + ".nz", nz);
    }
}

void exportAll(GridHandle& h)
{
    GridBuilder& b = h.builder;
    h.levels.assign(b.numberOfLevels(), Exported());
    for (int level = 0; level < b.numberOfLevels(); ++level) {
        Exported& E = h.levels[level];
        const LevelGrid& g = b.grid(level);
        std::vector<double> cx, cy, cz;
        std::vector<uint32_t> nbx, nby, nbz, nbn, geo;
        g.nodeValues(cx, cy, cz, nbx, nby, nbz, nbn, geo);
        E.put("coordX", cx);
        E.put("coordY", cy);
        E.put("coordZ", cz);
        E.put("neighborX", nbx);
        E.put("neighborY", nby);
        E.put("neighborZ", nbz);
        E.put("neighborNeg", nbn);
        E.put("geo", geo);
        E.put("dims", std::vector<int32_t> { (int32_t)g.nx, (int32_t)g.ny, (int32_t)g.nz });
        E.put("fluid", g.fluidNodes);
        concatenate(b.velocityBCs(level), E, "velocity", true, false);
        concatenate(b.slipBCs(level), E, "slip", false, true);
        // LevelGridBuilder::getStressValues / getStressQs (LevelGridBuilder.cpp:549-598)
        concatenate(b.stressBCs(level), E, "stress", false, true);
        {
            std::vector<int32_t> kN, off;
            std::vector<double> z0;
            for (const auto& l : b.stressBCs(level)) {
                kN.insert(kN.end(), l.kN.begin(), l.kN.end());
                off.insert(off.end(), l.samplingOffset.begin(), l.samplingOffset.end());
                z0.insert(z0.end(), l.z0.begin(), l.z0.end());
            }
            E.put("stress.kN", kN);
            E.put("stress.samplingOffset", off);
            E.put("stress.z0", z0);
        }
        std::vector<int32_t> gk;
        std::vector<double> gq;
        if (b.hasGeometryBC())
            g.geometryList(gk, gq);
        E.put("geometry.k", gk);
        E.put("geometry.q", gq);
        if (b.hasGeometryValues()) {
            const auto& v = b.geometryVelocity();
            E.put("geometry.vx", std::vector<double>(gk.size(), v[0]));
            E.put("geometry.vy", std::vector<double>(gk.size(), v[1]));
            E.put("geometry.vz", std::vector<double>(gk.size(), v[2]));
        }
        const auto& pres = b.pressureBCs(level);
        E.put("pressure.count", std::vector<int32_t> { (int32_t)pres.size() });
        for (size_t i = 0; i < pres.size(); ++i) {
            const std::string p = "pressure" + std::to_string(i);
            E.put(p + ".k", pres[i].k);
            E.put(p + ".kN", pres[i].kN);
            E.put(p + ".rho", pres[i].rho);
            E.put(p + ".q", pres[i].q);
            E.put(p + ".dir", std::vector<int32_t> { pres[i].d3q27Direction });
        }
        if (level + 1 < b.numberOfLevels()) {
            // LevelGridBuilder::getGridInterfaceIndices (+1 shifted sparse
            // indices) and getOffsetCF / getOffsetFC (the negated offset
            // direction, LevelGridBuilder.cpp:400-422)
            for (const char* tag : { "cf", "fc" }) {
                const InterfaceCells& ic = tag[0] == 'c' ? g.cf : g.fc;
                std::vector<uint32_t> c(ic.size()), f(ic.size());
                std::vector<double> ox(ic.size()), oy(ic.size()), oz(ic.size());
                for (size_t i = 0; i < ic.size(); ++i) {
                    c[i] = (uint32_t)(ic.coarse[i] + 1);
                    f[i] = (uint32_t)(ic.fine[i] + 1);
                    ox[i] = -(double)vfb::cx(ic.offset[i]);
                    oy[i] = -(double)vfb::cy(ic.offset[i]);
                    oz[i] = -(double)vfb::cz(ic.offset[i]);
                }
                const std::string t(tag);
                E.put(t + ".coarse", c);
                E.put(t + ".fine", f);
                E.put(t + ".offX", ox);
                E.put(t + ".offY", oy);
                E.put(t + ".offZ", oz);
            }
        }
    }
}
} // namespace

extern "C" {

/*
 * spec: [0..6] coarse grid start x,y,z, end x,y,z, delta; [7..9] periodic;
 * [10] refinement box present, [11..16] the box (min x,y,z, max x,y,z);
 * [17..18] layers fine / between levels (used when [17] > 0); [19] solid
 * primitive: 1 cuboid with [20..25] its extent, 2 sphere with [20..23]
 * centre and radius, 3 cylinder with [20..25] centre, radius, height, axis,
 * 4 vertical cylinder with [20..24] centre, radius, height, 5 conglomerate
 * ([62] parts added, [63] parts subtracted, 7 values each from [64] on:
 * kind 1..4 and its parameters);
 * [26..29] geometry BC (type 1 = no-slip, 2 = velocity with [27..29]); [30..59] six side BCs (side, type, v0, v1, v2) in the order they
 * are set, type 0 none, 1 no-slip, 2 velocity, 3 pressure, 4 slip (v = normal),
 * 5 stress (v = normal, with [176 + 3 i .. 178 + 3 i] the sampling offset,
 * z0 and the level-0 dx of side slot i; n >= 194); [60] enableThinWalls; [61]
 * finest level of the refinement box (0 = 1; n >= 62 values).  Same layout as
 * the grid oracle.  Returns NULL on error (see vfb_last_error).
 */
void* vfb_grid_build(const double* s, int n)
{
    vfb::clearError();
    if (!s || n < 61) {
        vfb::setError(VFB_ERR_INVALID_ARGUMENT, "grid spec needs 61 values");
        return nullptr;
    }
    auto* h = new GridHandle;
    try {
        h->builder.addCoarseGrid(s[0], s[1], s[2], s[3], s[4], s[5], s[6]);
        if (s[17] > 0)
            h->builder.setNumberOfLayers((uint32_t)s[17], (uint32_t)s[18]);
        if (s[10] > 0) {
            const int levelFine = (n > 61 && s[61] > 0) ? (int)s[61] : 1;
            h->builder.addGrid(Box { s[11], s[12], s[13], s[14], s[15], s[16] }, levelFine);
        }
        if (s[19] == 5) {
            // Conglomerate (Conglomerate.cpp:153-164): [62] parts added, [63]
            // parts subtracted, each 7 values from [64] on, added ones first
            if (n < 64)
                throw std::invalid_argument("a conglomerate needs the part counts at [62] and [63]");
            const int nAdd = (int)s[62], nSub = (int)s[63];
            if (nAdd < 1 || nSub < 0 || nAdd + nSub > 16 || n < 64 + 7 * (nAdd + nSub))
                throw std::invalid_argument("conglomerate part counts do not fit the spec");
            Solid solid;
            solid.kind = Solid::Kind::Conglomerate;
            for (int i = 0; i < nAdd + nSub; ++i) {
                const double* p = s + 64 + 7 * i;
                if (p[0] < 1 || p[0] > 4)
                    throw std::invalid_argument("a conglomerate part must be a primitive (kind 1..4)");
                (i < nAdd ? solid.add : solid.subtract).push_back(primitiveFrom(p));
            }
            h->builder.addGeometry(solid);
        } else if (s[19] > 0) {
            h->builder.addGeometry(primitiveFrom(s + 19));
        }
        h->builder.setPeriodicBoundaryCondition(s[7] > 0, s[8] > 0, s[9] > 0);
        h->builder.buildGrids(s[60] > 0);
        for (int i = 0; i < 6; ++i) {
            const double* b = s + 30 + 5 * i;
            applyBC(h->builder, (int)b[0], (int)b[1], b[2], b[3], b[4],
                    n >= kSpecWithStress ? s + kStressBase + 3 * i : nullptr);
        }
        if (s[19] > 0 && (int)s[26] != 0) {
            if ((int)s[26] == 2)
                h->builder.setVelocityGeometryBoundaryCondition(s[27], s[28], s[29]);
            else if ((int)s[26] == 1)
                h->builder.setNoSlipGeometryBoundaryCondition();
            else
                throw std::invalid_argument("only no-slip and velocity boundary conditions are supported on the geometry");
        }
        for (int level = 0; level < h->builder.numberOfLevels(); ++level)
            h->builder.grid(level).findFluidNodes();
        exportAll(*h);
    } catch (const std::exception& e) {
        vfb::setError(VFB_ERR_CONFIGURATION, "grid build failed: %s", e.what());
        delete h;
        return nullptr;
    }
    return h;
}

/*
 * The q values the builder gives a node on domain side `side` (0..5 = MX PX MY
 * PY MZ PZ) when every node around it is a boundary stopper and the sides
 * alreadySet[0..nSet) were set on it before (Side::setQs with its diagonal
 * reset, Side.cpp:149-215): q27[d] = 1/2 for the links along the side's
 * normal, -1 otherwise.  A check hook; the geometry side has no normal and
 * is rejected, as the reference rejects it.
 */
int vfb_debug_side_qs(int side, const int* alreadySet, int nSet, double* q27)
{
    vfb::clearError();
    if (side < 0 || side > 5 || !q27 || nSet < 0 || nSet > 6 || (nSet > 0 && !alreadySet))
        return vfb::setError(VFB_ERR_INVALID_ARGUMENT, "side must be 0..5 with up to six sides set before");
    LevelGrid g(0, 0, 0, 2, 2, 2, 1.0, 0);
    g.field.assign(g.size, STOPPER_OUT_OF_GRID_BOUNDARY);
    for (int i = 0; i < nSet; ++i) {
        if (alreadySet[i] < 0 || alreadySet[i] > 5)
            return vfb::setError(VFB_ERR_INVALID_ARGUMENT, "side %d set before has no normal", alreadySet[i]);
        g.bcAlreadySet.push_back((SideType)alreadySet[i]);
    }
    g.sideQs((SideType)side, 1, 1, 1, q27);
    return VFB_OK;
}

int vfb_grid_levels(void* h) { return h ? (int)static_cast<GridHandle*>(h)->levels.size() : 0; }

long long vfb_grid_count(void* h, int level, const char* name)
{
    auto* H = static_cast<GridHandle*>(h);
    if (!H || !name || level < 0 || level >= (int)H->levels.size())
        return -1;
    auto it = H->levels[level].data.find(name);
    if (it == H->levels[level].data.end())
        return -1;
    return (long long)(it->second.size() / H->levels[level].elem[name]);
}

int vfb_grid_elem_size(void* h, int level, const char* name)
{
    auto* H = static_cast<GridHandle*>(h);
    if (!H || !name || level < 0 || level >= (int)H->levels.size())
        return -1;
    auto it = H->levels[level].elem.find(name);
    return it == H->levels[level].elem.end() ? -1 : it->second;
}

int vfb_grid_copy(void* h, int level, const char* name, void* out)
{
    auto* H = static_cast<GridHandle*>(h);
    if (!H || !name || level < 0 || level >= (int)H->levels.size())
        return VFB_ERR_INVALID_ARGUMENT;
    auto it = H->levels[level].data.find(name);
    if (it == H->levels[level].data.end())
        return VFB_ERR_INVALID_ARGUMENT;
    if (!it->second.empty()) {
        if (!out)
            return VFB_ERR_INVALID_ARGUMENT;
        std::memcpy(out, it->second.data(), it->second.size());
    }
    return VFB_OK;
}

void vfb_grid_free(void* h) { delete static_cast<GridHandle*>(h); }

void* vfb_grid_create(int levels)
{
    vfb::clearError();
    if (levels < 1 || levels > 32) {
        vfb::setError(VFB_ERR_INVALID_ARGUMENT, "levels %d outside [1, 32]", levels);
        return nullptr;
    }
    auto* h = new GridHandle;
    h->levels.assign((size_t)levels, Exported());
    return h;
}

int vfb_grid_put(void* h, int level, const char* name, int elemSize, long long count, const void* data)
{
    vfb::clearError();
    auto* H = static_cast<GridHandle*>(h);
    if (!H || !name || level < 0 || level >= (int)H->levels.size())
        return vfb::setError(VFB_ERR_INVALID_ARGUMENT, "no grid level %d", level);
    if (!(elemSize == 1 || elemSize == 2 || elemSize == 4 || elemSize == 8) || count < 0 || (count > 0 && !data))
        return vfb::setError(VFB_ERR_INVALID_ARGUMENT, "array %s: element size %d, count %lld", name, elemSize, count);
    std::vector<char>& d = H->levels[level].data[name];
    d.resize((size_t)count * (size_t)elemSize);
    if (count > 0)
        std::memcpy(d.data(), data, d.size());
    H->levels[level].elem[name] = elemSize;
    return VFB_OK;
}

} // extern "C"
