// ref_grid.cpp -- harness around the reference's grid builder.
//
// TEST INFRASTRUCTURE ONLY (oracle).  Builds a grid with the reference's own
// MultipleGridBuilder / LevelGridBuilder (src/gpu/GridGenerator, compiled by
// oracle/Makefile with a no-op logging stand-in) and exposes every array the
// GPU data-structure initializer reads from it
// (src/gpu/core/DataStructureInitializer/GridReaderGenerator/GridGenerator.cpp:91-1035),
// so that the repository's grid builder can be compared with it element by element.
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include <basics/DataTypes.h>

#include "geometries/Cuboid/Cuboid.h"
#include "geometries/Sphere/Sphere.h"
#include "geometries/Cylinder/Cylinder.h"
#include "geometries/VerticalCylinder/VerticalCylinder.h"
#include "geometries/Conglomerate/Conglomerate.h"
#include "grid/BoundaryConditions/Side.h"
#include "grid/GridBuilder/LevelGridBuilder.h"
#include "grid/GridBuilder/MultipleGridBuilder.h"
#include "grid/Grid.h"

namespace
{
struct Arrays {
    std::map<std::string, std::vector<char>> data; // raw bytes
    std::map<std::string, int> elemSize;
    template <typename T>
    void put(const std::string& name, const T* p, size_t n)
    {
        std::vector<char>& v = data[name];
        v.resize(n * sizeof(T));
        if (n)
            std::memcpy(v.data(), p, n * sizeof(T));
        elemSize[name] = (int)sizeof(T);
    }
};
struct Handle {
    std::vector<Arrays> levels;
};

SideType sideOf(int s)
{
    switch (s) {
    case 0: return SideType::MX;
    case 1: return SideType::PX;
    case 2: return SideType::MY;
    case 3: return SideType::PY;
    case 4: return SideType::MZ;
    case 5: return SideType::PZ;
    default: return SideType::GEOMETRY;
    }
}

void applyBC(LevelGridBuilder& b, SideType side, int type, double v0, double v1, double v2,
             const double* stress = nullptr)
{
    switch (type) {
    case 1: b.setNoSlipBoundaryCondition(side); break;
    case 2: b.setVelocityBoundaryCondition(side, (real)v0, (real)v1, (real)v2); break;
    case 3: b.setPressureBoundaryCondition(side, (real)v0); break;
    case 4: b.setSlipBoundaryCondition(side, (real)v0, (real)v1, (real)v2); break;
    case 5:
        b.setStressBoundaryCondition(side, (real)v0, (real)v1, (real)v2, (uint)stress[0], (real)stress[1],
                                     (real)stress[2]);
        break;
    default: break;
    }
}

void exportQs(Arrays& A, const std::string& name, uint n, void (LevelGridBuilder::*get)(real* [27], int) const,
              LevelGridBuilder& b, int level)
{
    std::vector<real> q(27 * (size_t)n, (real)-1);
    real* qs[27];
    for (int d = 0; d < 27; ++d)
        qs[d] = q.data() + (size_t)d * n;
    if (n)
        (b.*get)(qs, level);
    A.put(name, q.data(), q.size());
}
} // namespace

#ifdef VF_DOUBLE_ACCURACY
#define REF(name) name##_f64
#else
#define REF(name) name##_f32
#endif

extern "C" {

// spec (doubles):
//  [0..6]   coarse grid start x,y,z, end x,y,z, delta (addCoarseGrid arguments)
//  [7..9]   periodic x, y, z
//  [10]     number of refinement boxes (0 or 1), [11..16] the box (Cuboid, level 1)
//  [17..18] number of layers fine / between levels (used when [17] > 0)
//  [19]     solid primitive: 1 Cuboid with [20..25] its extent, 2 Sphere with [20..23]
//           centre and radius, 3 Cylinder with [20..25] centre, radius, height and
//           axis (0 x, 1 y, 2 z), 4 VerticalCylinder with [20..24] centre, radius and
//           height, 5 Conglomerate of [62] added and [63] subtracted primitives,
//           7 values each (kind 1..4 and the parameters above) from [64] on
//  [26..29] geometry BC type (1 no-slip, 2 velocity, 4 slip) and values
//  [30..59] six side BCs in the order they are set: side id (0..5 = MX..PZ),
//           type (0 none, 1 no-slip, 2 velocity, 3 pressure, 4 slip, 5 stress), 3 values
//  [176 + 3 i .. 178 + 3 i]  stress side slot i: sampling offset, z0, level-0 dx
//           (present when a slot has type 5)
//  [60]     enableThinWalls argument of buildGrids
//  [61]     finest level of the refinement box (0 = level 1)
// a primitive from 7 spec values: kind (1 Cuboid, 2 Sphere, 3 Cylinder,
// 4 VerticalCylinder) and its parameters
static std::shared_ptr<Object> primitive(const double* p)
{
    if (p[0] == 4)
        return std::make_shared<VerticalCylinder>(p[1], p[2], p[3], p[4], p[5]);
    if (p[0] == 3)
        return std::make_shared<Cylinder>(p[1], p[2], p[3], p[4], p[5], (Axis)(int)p[6]);
    if (p[0] == 2)
        return std::make_shared<Sphere>(p[1], p[2], p[3], p[4]);
    return std::make_shared<Cuboid>(p[1], p[2], p[3], p[4], p[5], p[6]);
}

void* REF(vfref_grid_build)(const double* s)
{
    auto builder = std::make_shared<MultipleGridBuilder>();
    builder->addCoarseGrid((real)s[0], (real)s[1], (real)s[2], (real)s[3], (real)s[4], (real)s[5], (real)s[6]);
    if (s[17] > 0)
        builder->setNumberOfLayers((uint)s[17], (uint)s[18]);
    if (s[10] > 0)
        builder->addGrid(std::make_shared<Cuboid>(s[11], s[12], s[13], s[14], s[15], s[16]),
                         s[61] > 0 ? (uint)s[61] : 1u);
    if (s[19] == 5) {
        auto conglomerate = Conglomerate::makeShared();
        const int nAdd = (int)s[62], nSub = (int)s[63];
        for (int i = 0; i < nAdd + nSub; ++i) {
            auto part = primitive(s + 64 + 7 * i);
            if (i < nAdd)
                conglomerate->add(part);
            else
                conglomerate->subtract(part);
        }
        builder->addGeometry(conglomerate);
    } else if (s[19] > 0) {
        builder->addGeometry(primitive(s + 19));
    }
    builder->setPeriodicBoundaryCondition(s[7] > 0, s[8] > 0, s[9] > 0);
    builder->buildGrids(s[60] > 0);

    for (int i = 0; i < 6; ++i) {
        const double* b = s + 30 + 5 * i;
        if ((int)b[1] != 0)
            applyBC(*builder, sideOf((int)b[0]), (int)b[1], b[2], b[3], b[4], s + 176 + 3 * i);
    }
    if (s[19] > 0 && (int)s[26] != 0)
        applyBC(*builder, SideType::GEOMETRY, (int)s[26], s[27], s[28], s[29]);

    builder->findFluidNodes(false);

    auto* h = new Handle;
    const uint numberOfLevels = builder->getNumberOfGridLevels();
    h->levels.resize(numberOfLevels);
    for (uint level = 0; level < numberOfLevels; ++level) {
        Arrays& A = h->levels[level];
        const uint N = builder->getNumberOfNodes(level) + 1;
        std::vector<real> cx(N), cy(N), cz(N);
        std::vector<uint> nx(N), ny(N), nz(N), nn(N), geo(N);
        builder->getNodeValues(cx.data(), cy.data(), cz.data(), nx.data(), ny.data(), nz.data(), nn.data(), geo.data(),
                               level);
        A.put("coordX", cx.data(), N);
        A.put("coordY", cy.data(), N);
        A.put("coordZ", cz.data(), N);
        A.put("neighborX", nx.data(), N);
        A.put("neighborY", ny.data(), N);
        A.put("neighborZ", nz.data(), N);
        A.put("neighborNeg", nn.data(), N);
        A.put("geo", geo.data(), N);
        int dims[3];
        builder->getDimensions(dims[0], dims[1], dims[2], level);
        A.put("dims", dims, 3);

        const uint nf = builder->getNumberOfFluidNodes(level);
        std::vector<uint> fluid(nf);
        if (nf)
            builder->getFluidNodeIndices(fluid.data(), level);
        A.put("fluid", fluid.data(), nf);

        const uint nv = builder->getVelocitySize(level);
        std::vector<int> vk(nv);
        std::vector<real> vx(nv), vy(nv), vz(nv);
        if (nv)
            builder->getVelocityValues(vx.data(), vy.data(), vz.data(), vk.data(), level);
        A.put("velocity.k", vk.data(), nv);
        A.put("velocity.vx", vx.data(), nv);
        A.put("velocity.vy", vy.data(), nv);
        A.put("velocity.vz", vz.data(), nv);
        exportQs(A, "velocity.q", nv, &LevelGridBuilder::getVelocityQs, *builder, level);

        const uint ns = builder->getSlipSize(level);
        std::vector<int> sk(ns);
        std::vector<real> snx(ns), sny(ns), snz(ns);
        if (ns)
            builder->getSlipValues(snx.data(), sny.data(), snz.data(), sk.data(), level);
        A.put("slip.k", sk.data(), ns);
        A.put("slip.nx", snx.data(), ns);
        A.put("slip.ny", sny.data(), ns);
        A.put("slip.nz", snz.data(), ns);
        exportQs(A, "slip.q", ns, &LevelGridBuilder::getSlipQs, *builder, level);

        const uint nt = builder->getStressSize(level);
        {
            std::vector<int> tk(nt), tkN(nt), toff(nt);
            std::vector<real> tnx(nt), tny(nt), tnz(nt), v(nt), z0(nt);
            if (nt)
                builder->getStressValues(tnx.data(), tny.data(), tnz.data(), v.data(), v.data(), v.data(), v.data(),
                                         v.data(), v.data(), tk.data(), tkN.data(), toff.data(), z0.data(), level);
            A.put("stress.k", tk.data(), nt);
            A.put("stress.kN", tkN.data(), nt);
            A.put("stress.nx", tnx.data(), nt);
            A.put("stress.ny", tny.data(), nt);
            A.put("stress.nz", tnz.data(), nt);
            A.put("stress.samplingOffset", toff.data(), nt);
            A.put("stress.z0", z0.data(), nt);
            exportQs(A, "stress.q", nt, &LevelGridBuilder::getStressQs, *builder, level);
        }

        const uint ng = builder->getGeometrySize(level);
        std::vector<int> gk(ng);
        if (ng)
            builder->getGeometryIndices(gk.data(), level);
        A.put("geometry.k", gk.data(), ng);
        exportQs(A, "geometry.q", ng, &LevelGridBuilder::getGeometryQs, *builder, level);
        // hasGeometryValues() is also true after a no-slip geometry BC
        // (LevelGridBuilder.cpp:287-289), whose velocity lists stay empty, so
        // reading them would run past their end: values only for a velocity
        if (builder->hasGeometryValues() && (int)s[26] == 2) {
            std::vector<real> gvx(ng), gvy(ng), gvz(ng);
            if (ng)
                builder->getGeometryValues(gvx.data(), gvy.data(), gvz.data(), level);
            A.put("geometry.vx", gvx.data(), ng);
            A.put("geometry.vy", gvy.data(), ng);
            A.put("geometry.vz", gvz.data(), ng);
        }

        const size_t npb = builder->getNumberOfPressureBoundaryConditions(level);
        int npbi = (int)npb;
        A.put("pressure.count", &npbi, 1);
        for (size_t i = 0; i < npb; ++i) {
            const size_t n = builder->getSizeOfPressureBoundaryCondition(level, (uint)i);
            std::vector<int> k(n), kN(n);
            std::vector<real> rho(n);
            std::vector<real> q(27 * n, (real)-1);
            real* qs[27];
            for (int d = 0; d < 27; ++d)
                qs[d] = q.data() + (size_t)d * n;
            if (n) {
                builder->getPressureValues(rho.data(), k.data(), kN.data(), level, (uint)i);
                builder->getPressureQs(qs, level, (uint)i);
            }
            const std::string p = "pressure" + std::to_string(i);
            A.put(p + ".k", k.data(), n);
            A.put(p + ".kN", kN.data(), n);
            A.put(p + ".rho", rho.data(), n);
            A.put(p + ".q", q.data(), q.size());
            int dir = (int)builder->getPressureBoundaryConditionDirection(level, (uint)i);
            A.put(p + ".dir", &dir, 1);
        }

        if (level + 1 < numberOfLevels) {
            const uint ncf = builder->getNumberOfNodesCF(level);
            const uint nfc = builder->getNumberOfNodesFC(level);
            std::vector<uint> cfc(ncf), cff(ncf), fcc(nfc), fcf(nfc);
            builder->getGridInterfaceIndices(cfc.data(), cff.data(), fcc.data(), fcf.data(), level);
            std::vector<real> ox(ncf), oy(ncf), oz(ncf), px(nfc), py(nfc), pz(nfc);
            builder->getOffsetCF(ox.data(), oy.data(), oz.data(), level);
            builder->getOffsetFC(px.data(), py.data(), pz.data(), level);
            A.put("cf.coarse", cfc.data(), ncf);
            A.put("cf.fine", cff.data(), ncf);
            A.put("fc.coarse", fcc.data(), nfc);
            A.put("fc.fine", fcf.data(), nfc);
            A.put("cf.offX", ox.data(), ncf);
            A.put("cf.offY", oy.data(), ncf);
            A.put("cf.offZ", oz.data(), ncf);
            A.put("fc.offX", px.data(), nfc);
            A.put("fc.offY", py.data(), nfc);
            A.put("fc.offZ", pz.data(), nfc);
        }
    }
    return h;
}

int REF(vfref_grid_levels)(void* h) { return (int)static_cast<Handle*>(h)->levels.size(); }

// number of elements of an exported array, -1 if absent
long long REF(vfref_grid_count)(void* h, int level, const char* name)
{
    Handle* H = static_cast<Handle*>(h);
    if (level < 0 || level >= (int)H->levels.size())
        return -1;
    auto it = H->levels[level].data.find(name);
    if (it == H->levels[level].data.end())
        return -1;
    return (long long)(it->second.size() / H->levels[level].elemSize[name]);
}

int REF(vfref_grid_elem_size)(void* h, int level, const char* name)
{
    Handle* H = static_cast<Handle*>(h);
    auto it = H->levels[level].elemSize.find(name);
    return it == H->levels[level].elemSize.end() ? -1 : it->second;
}

int REF(vfref_grid_copy)(void* h, int level, const char* name, void* out)
{
    Handle* H = static_cast<Handle*>(h);
    auto it = H->levels[level].data.find(name);
    if (it == H->levels[level].data.end())
        return -1;
    if (!it->second.empty())
        std::memcpy(out, it->second.data(), it->second.size());
    return 0;
}

void REF(vfref_grid_free)(void* h) { delete static_cast<Handle*>(h); }

} // extern "C"
