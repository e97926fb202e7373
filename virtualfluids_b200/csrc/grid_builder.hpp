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

enum class BCKind { NoSlip = 1, Velocity = 2, Pressure = 3, Slip = 4 };

struct Box {
    double minX, minY, minZ, maxX, maxY, maxZ;
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
    std::vector<double> normalX, normalY, normalZ; // slip normals per node
    size_t size() const { return k.size(); }
};

class LevelGrid
{
public:
    LevelGrid(double startX, double startY, double startZ, double endX, double endY, double endZ, double delta,
              int level);

    // --- construction (mirrors GridImp::inital / findSparseIndices) ------
    void initialNodes();
    void findStoppers();
    void findSparseIndices();
    void findFluidNodes();

    // --- accessors --------------------------------------------------------
    uint32_t nx, ny, nz;
    uint64_t size;
    double startX, startY, startZ, endX, endY, endZ, delta;
    int level;
    bool periodic[3] = { false, false, false };

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
    bool isFluid(uint64_t idx) const;
    bool isStopper(uint64_t idx) const;
    bool isStopperForBC(int64_t idx) const;
    bool hasNeighborOfType(uint64_t idx, uint8_t type) const;
    bool hasAllNeighbors(uint64_t idx) const;
    // q values of a node on a domain side (Side::setQs)
    void sideQs(SideType side, int64_t ix, int64_t iy, int64_t iz, double* qNode) const;

private:
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
    void setPeriodicBoundaryCondition(bool px, bool py, bool pz);
    void buildGrids(bool enableThinWalls = false);

    void setNoSlipBoundaryCondition(SideType side);
    void setVelocityBoundaryCondition(SideType side, double vx, double vy, double vz);
    void setPressureBoundaryCondition(SideType side, double rho);
    void setSlipBoundaryCondition(SideType side, double normalX, double normalY, double normalZ);

    int numberOfLevels() const { return (int)grids.size(); }
    LevelGrid& grid(int level) { return *grids.at(level); }
    const LevelGrid& grid(int level) const { return *grids.at(level); }

    // concatenated lists per level in the order the reference exports them
    // (LevelGridBuilder::getVelocityValues etc.)
    const std::vector<BCList>& velocityBCs(int level) const { return velocity.at(level); }
    const std::vector<BCList>& slipBCs(int level) const { return slip.at(level); }
    const std::vector<BCList>& pressureBCs(int level) const { return pressure.at(level); }

private:
    std::vector<std::unique_ptr<LevelGrid>> grids;
    std::vector<std::vector<BCList>> velocity, slip, pressure;
    bool built = false;
};

} // namespace vfb::grid
