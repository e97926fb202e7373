// grid_builder.hpp -- host-side construction of the sparse lattice, its
// neighbour arrays, fluid-node list and boundary-condition lists.
//
// Produces, element for element, the arrays VirtualFluids' GridGenerator
// hands to the GPU solver (src/gpu/GridGenerator/grid/GridImp.cpp:914-1121,
// 2146-2185; grid/BoundaryConditions/Side.cpp:64-404;
// grid/GridBuilder/LevelGridBuilder.cpp:395-944): the same node numbering
// (x fastest, node 0 a dummy, +1 shift), the same stopper layer around the
// domain, the same periodic wiring and the same q-value placement on the
// domain sides.  The builder works on integer node indices; the reference
// works on floating-point coordinates mapped back to indices, which is the
// same mapping for every node of the grid.
#pragma once

#include <array>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

namespace vfb::grid
{

// node states (src/gpu/GridGenerator/grid/NodeValues.h)
enum NodeType : uint8_t {
    FLUID = 0,
    FLUID_CFC = 1,
    FLUID_CFF = 2,
    FLUID_FCC = 3,
    FLUID_FCF = 4,
    BC_PRESSURE = 20,
    BC_VELOCITY = 21,
    BC_SOLID = 22,
    BC_SLIP = 23,
    BC_NOSLIP = 24,
    BC_OUTFLOW = 25,
    BC_STRESS = 26,
    STOPPER_OUT_OF_GRID = 30,
    STOPPER_COARSE_UNDER_FINE = 31,
    STOPPER_SOLID = 32,
    STOPPER_OUT_OF_GRID_BOUNDARY = 33,
    INVALID_OUT_OF_GRID = 40,
    INVALID_COARSE_UNDER_FINE = 41,
    INVALID_SOLID = 42,
    OVERLAP_TMP = 60,
};

enum class SideType { MX = 0, PX = 1, MY = 2, PY = 3, MZ = 4, PZ = 5, GEOMETRY = 6 };

enum class BCKind { NoSlip = 1, Velocity = 2, Pressure = 3, Slip = 4, Stress = 5 };

struct Box {
    double minX, minY, minZ, maxX, maxY, maxZ;
    // Cuboid::isPointInObject (Cuboid.cpp): strictly inside, with the
    // reference's relative comparison tolerance (FLT_EPSILON)
    bool containsPoint(double x, double y, double z) const;
};

// A solid geometric primitive of the reference (geometries/Cuboid,
// geometries/Sphere): which lattice points it holds and, for the sphere, where
// a ray from a point along a lattice direction meets its surface.
struct Solid {
    enum class Kind { Cuboid, Sphere, Cylinder, Conglomerate } kind = Kind::Cuboid;
    Box box {};                           // cuboid
    double cx = 0, cy = 0, cz = 0, r = 0; // sphere, cylinder (centre, radius)
    double height = 0;                    // cylinder: length along its axis
    int axis = 0;                         // cylinder: 0 x, 1 y, 2 z
    std::vector<Solid> add, subtract;     // conglomerate: primitives united, then removed
    bool contains(double x, double y, double z) const;
    // Object::getIntersection: true with t (in units of the direction
    // vector) when the ray point + t * direction meets the surface at t >= 0;
    // a cuboid, cylinder or conglomerate reports no intersection, as the
    // reference's objects do
    bool intersect(double px, double py, double pz, double dx, double dy, double dz, double& t) const;
};

// interface cells between a level and the next finer one
// (GridInterface::cf / fc): matrix indices until the sparse renumbering,
// sparse indices after it; offset = index of the D3Q27 direction
struct InterfaceCells {
    std::vector<int64_t> coarse, fine;
    std::vector<int> offset;
    size_t size() const { return coarse.size(); }
};

// One compacted boundary-condition list of one level, in the GPU layout of
// QforBoundaryConditions (src/gpu/core/Calculation/Calculation.h:105-117):
// node indices (+1 shifted), q direction-major (q[d * n + i]).
struct BCList {
    BCKind kind;
    SideType side;
    int d3q27Direction = 0;             // pressure: outward normal as a D3Q27 id
    std::vector<int32_t> k;
    std::vector<int32_t> kN;            // pressure: neighbour inside the domain
    std::vector<double> q;              // 27 * size, -1 = no link
    std::vector<double> vx, vy, vz;     // velocity per node
    std::vector<double> rho;            // pressure per node
    std::vector<double> normalX, normalY, normalZ; // slip and stress normals per node
    std::vector<int32_t> samplingOffset; // stress: sampling height in nodes (kN holds the sampling node)
    std::vector<double> z0;              // stress: roughness length in this level's lattice units
    size_t size() const { return k.size(); }
};

class LevelGrid
{
public:
    LevelGrid(double startX, double startY, double startZ, double endX, double endY, double endZ, double delta,
              int level);

    // --- construction (mirrors GridImp::inital / findSparseIndices) ------
    // node types of the level: inner region (from the refinement box, or
    // from the finer level for intermediate levels), overlap layers, odd
    // cells completed, end-of-grid stoppers
    void initial(const LevelGrid* finer);
    void findSparseIndices();
    void findFluidNodes();
    // solid primitive on this level (GridImp::mesh + findQsPrimitive for a
    // geometric primitive): inside nodes removed, one stopper layer inside the
    // solid, one BC_SOLID layer outside it, the links' q values
    void meshSolid(const Solid& solid, bool thinWalls);
    // interface cells to the next finer level (GridImp::findGridInterface,
    // repairGridInterfaceOnMultiGPU) and their sparse renumbering
    void findGridInterface(LevelGrid& fine);
    void repairGridInterface(const LevelGrid& fine);
    void renumberGridInterface(const LevelGrid& fine);

    // --- accessors --------------------------------------------------------
    uint32_t nx, ny, nz;
    uint64_t size;
    double startX, startY, startZ, endX, endY, endZ, delta;
    int level;
    bool periodic[3] = { false, false, false };
    bool oddStart[3] = { false, false, false };
    uint32_t numberOfLayers = 0;    // overlap layers around the inner region
    bool innerFromFiner = false;    // intermediate level: inner region from the finer level
    bool hasShape = false;          // level > 0: the refinement box
    Box shape {};
    std::vector<int64_t> solidBoundaryIndex; // BC_SOLID nodes in matrix order, -1 elsewhere
    uint32_t numberOfSolidBoundaryNodes = 0;
    std::vector<double> solidQ;             // q[d * numberOfSolidBoundaryNodes + BC_SOLID number], -1 none
    InterfaceCells cf, fc;          // to the next finer level

    std::vector<uint8_t> field;
    std::vector<int64_t> sparseIndex;       // -1 for removed nodes
    uint64_t sparseSize = 0;
    std::vector<int64_t> neighborX, neighborY, neighborZ, neighborNeg; // sparse, -1 none
    std::vector<uint32_t> fluidNodes;       // +1 shifted sparse indices
    std::vector<SideType> bcAlreadySet;

    // GPU arrays (+1 shifted, node 0 dummy)
    void nodeValues(std::vector<double>& cx, std::vector<double>& cy, std::vector<double>& cz,
                    std::vector<uint32_t>& nbx, std::vector<uint32_t>& nby, std::vector<uint32_t>& nbz,
                    std::vector<uint32_t>& nbneg, std::vector<uint32_t>& geo) const;

    int64_t index(int64_t ix, int64_t iy, int64_t iz) const
    {
        if (ix < 0 || iy < 0 || iz < 0 || ix >= (int64_t)nx || iy >= (int64_t)ny || iz >= (int64_t)nz)
            return -1;
        return ix + (int64_t)nx * (iy + (int64_t)ny * iz);
    }
    void coords(uint64_t idx, int64_t& ix, int64_t& iy, int64_t& iz) const
    {
        ix = (int64_t)(idx % nx);
        iy = (int64_t)((idx / nx) % ny);
        iz = (int64_t)((idx / nx) / ny % nz);
    }
    // coordinates of a matrix index and the matrix index of a coordinate
    // (GridImp::transIndexToCoords / transCoordToIndex: rounded to the
    // nearest node, -1 outside the grid)
    double coordX(int64_t ix) const { return (double)ix * delta + startX; }
    double coordY(int64_t iy) const { return (double)iy * delta + startY; }
    double coordZ(int64_t iz) const { return (double)iz * delta + startZ; }
    int64_t coordToIndex(double x, double y, double z) const;
    bool isFluid(uint64_t idx) const;
    bool isStopper(uint64_t idx) const;
    bool isStopperForBC(int64_t idx) const;
    bool hasNeighborOfType(uint64_t idx, uint8_t type) const;
    bool hasAllNeighbors(uint64_t idx) const;
    // q values of a node on a domain side (Side::setQs)
    void sideQs(SideType side, int64_t ix, int64_t iy, int64_t iz, double* qNode) const;

    // geometry boundary list of this level (Geometry::addIndices): BC_SOLID
    // nodes in matrix order, q = 1/2 towards stopper nodes, -1 otherwise
    void geometryList(std::vector<int32_t>& k, std::vector<double>& q) const;

private:
    void findInnerNodes();
    void setInnerBasedOnFinerGrid(const LevelGrid& fine);
    void addOverlap();
    void findStoppers();
    int64_t oddCellStart(int64_t i, int axis) const;
    bool cellContainsOnly(int64_t x0, int64_t y0, int64_t z0, uint8_t a, uint8_t b) const;
    void setNonStopperOutOfGridCellTo(uint64_t idx, uint8_t type);
    int64_t coarseToFineIndex(uint64_t idx, const LevelGrid& fine) const;
    int64_t fineToCoarseIndex(uint64_t idx, const LevelGrid& fine) const;
    bool isNeighborFineInvalid(int64_t ix, int64_t iy, int64_t iz, const LevelGrid& fine) const;
    int64_t offsetCellCF(uint64_t idx, int& offset) const;
    int64_t offsetCellFC(uint64_t idx, int& offset) const;
    int64_t neighborIndexPositive(int64_t ix, int64_t iy, int64_t iz, int axis) const;
    int64_t negativeNeighborIndex(int64_t ix, int64_t iy, int64_t iz) const;
    int64_t firstFluidAlong(int64_t ix, int64_t iy, int64_t iz, int axis) const;
    int64_t lastFluidAlong(int64_t ix, int64_t iy, int64_t iz, int axis) const;
    void fixOddCells();
};

// Multi-level builder facade (MultipleGridBuilder / LevelGridBuilder API).
class GridBuilder
{
public:
    void addCoarseGrid(double startX, double startY, double startZ, double endX, double endY, double endZ,
                       double delta);
    // refinement box up to level levelFine (MultipleGridBuilder::addGrid):
    // one grid per missing level, staggered on its parent, with the overlap
    // layers of setNumberOfLayers
    void addGrid(const Box& box, int levelFine);
    void setNumberOfLayers(uint32_t fine, uint32_t betweenLevels);
    // solid primitive, meshed on the finest level (MultipleGridBuilder::addGeometry)
    void addGeometry(const Solid& solid);
    void setPeriodicBoundaryCondition(bool px, bool py, bool pz);
    void buildGrids(bool enableThinWalls = false);

    void setNoSlipBoundaryCondition(SideType side);
    void setVelocityBoundaryCondition(SideType side, double vx, double vy, double vz);
    void setPressureBoundaryCondition(SideType side, double rho);
    void setSlipBoundaryCondition(SideType side, double normalX, double normalY, double normalZ);
    // wall-model BC (LevelGridBuilder::setStressBoundaryCondition, LevelGridBuilder.cpp:129-150):
    // the side's nodes with their normal, the node samplingOffset layers
    // further inside as the velocity sampling node, and z0 * 2^level / dx as
    // the level's roughness length
    void setStressBoundaryCondition(SideType side, double normalX, double normalY, double normalZ,
                                    uint32_t samplingOffset, double z0, double dx);
    // no-slip on the solid geometry's BC_SOLID nodes, every level
    void setNoSlipGeometryBoundaryCondition();
    void setVelocityGeometryBoundaryCondition(double vx, double vy, double vz);

    int numberOfLevels() const { return (int)grids.size(); }
    LevelGrid& grid(int level) { return *grids.at(level); }
    const LevelGrid& grid(int level) const { return *grids.at(level); }

    // concatenated lists per level in the order the reference exports them
    // (LevelGridBuilder::getVelocityValues etc.)
    const std::vector<BCList>& velocityBCs(int level) const { return velocity.at(level); }
    const std::vector<BCList>& slipBCs(int level) const { return slip.at(level); }
    const std::vector<BCList>& pressureBCs(int level) const { return pressure.at(level); }
    const std::vector<BCList>& stressBCs(int level) const { return stress.at(level); }
    bool hasGeometryBC() const { return geometryNoSlip; }
    // LevelGridBuilder::hasGeometryValues / getGeometryValues: a velocity on the geometry
    bool hasGeometryValues() const { return geometryHasValues; }
    const std::array<double, 3>& geometryVelocity() const { return geometryValues; }

private:
    std::array<double, 6> staggeredCoordinates(const Box& shape, int level, int levelFine, bool odd[3]) const;
    std::vector<std::unique_ptr<LevelGrid>> grids;
    std::vector<std::vector<BCList>> velocity, slip, pressure, stress;
    uint32_t layersFine = 12, layersBetweenLevels = 8; // MultipleGridBuilder.cpp:53
    bool hasSolid = false;
    Solid solid {};
    bool geometryNoSlip = false;
    bool geometryHasValues = false;
    std::array<double, 3> geometryValues { 0.0, 0.0, 0.0 };
    bool built = false;
};

} // namespace vfb::grid
