// grid_builder.cpp -- see grid_builder.hpp.
#include "grid_builder.hpp"

#include <cmath>
#include <stdexcept>

#include "d3q27.cuh"

namespace vfb::grid
{

namespace
{
// D3Q27 id of the outward normal of a side (Side.h sideToD3Q27)
int sideDirection(SideType s)
{
    switch (s) {
    case SideType::MX: return dM00;
    case SideType::PX: return dP00;
    case SideType::MY: return d0M0;
    case SideType::PY: return d0P0;
    case SideType::MZ: return d00M;
    case SideType::PZ: return d00P;
    default: return d000;
    }
}
int sideAxis(SideType s) { return (int)s / 2; }
int sideSign(SideType s) { return ((int)s % 2) ? 1 : -1; }

bool alignedWith(int dir, SideType s)
{
    const int c[3] = { cx(dir), cy(dir), cz(dir) };
    return sideSign(s) * c[sideAxis(s)] > 0;
}
} // namespace

LevelGrid::LevelGrid(double sx, double sy, double sz, double ex, double ey, double ez, double d, int lvl)
    : startX(sx), startY(sy), startZ(sz), endX(ex), endY(ey), endZ(ez), delta(d), level(lvl)
{
    // GridImp::initalNumberOfNodesAndSize (GridImp.cpp:107-119)
    nx = (uint32_t)std::lround((endX - startX + delta) / delta);
    ny = (uint32_t)std::lround((endY - startY + delta) / delta);
    nz = (uint32_t)std::lround((endZ - startZ + delta) / delta);
    size = (uint64_t)nx * ny * nz;
}

bool LevelGrid::isFluid(uint64_t i) const
{
    const uint8_t t = field[i];
    return t == FLUID || t == FLUID_CFC || t == FLUID_CFF || t == FLUID_FCC || t == FLUID_FCF || t == BC_SOLID ||
           t == BC_OUTFLOW || t == BC_VELOCITY || t == BC_PRESSURE || t == BC_SLIP || t == BC_STRESS;
}

bool LevelGrid::isStopper(uint64_t i) const
{
    const uint8_t t = field[i];
    return t == STOPPER_OUT_OF_GRID || t == STOPPER_COARSE_UNDER_FINE || t == STOPPER_SOLID ||
           t == STOPPER_OUT_OF_GRID_BOUNDARY;
}

bool LevelGrid::isStopperForBC(int64_t i) const
{
    if (i < 0)
        return false;
    const uint8_t t = field[(uint64_t)i];
    return t == STOPPER_OUT_OF_GRID_BOUNDARY || t == STOPPER_OUT_OF_GRID || t == STOPPER_SOLID;
}

// GridImp::hasNeighborOfType (GridImp.cpp:597-612): all 27 directions
bool LevelGrid::hasNeighborOfType(uint64_t idx, uint8_t type) const
{
    int64_t ix, iy, iz;
    coords(idx, ix, iy, iz);
    for (int d = 0; d < 27; ++d) {
        const int64_t n = index(ix + cx(d), iy + cy(d), iz + cz(d));
        if (n >= 0 && field[(uint64_t)n] == type)
            return true;
    }
    return false;
}

bool LevelGrid::hasAllNeighbors(uint64_t idx) const
{
    int64_t ix, iy, iz;
    coords(idx, ix, iy, iz);
    for (int d = 0; d < 27; ++d)
        if (index(ix + cx(d), iy + cy(d), iz + cz(d)) < 0)
            return false;
    return true;
}

// Coarse level: everything but the outermost layer is fluid
// (GridImp::findInnerNode, GridImp.cpp:225-248), then odd cells are completed
// (GridImp::fixOddCell, :466-472) and the outermost layer becomes the stopper
// layer (GridImp::findEndOfGridStopperNode, :436-448).
void LevelGrid::initialNodes()
{
    field.assign(size, INVALID_OUT_OF_GRID);
    for (uint32_t z = 1; z + 1 < nz; ++z)
        for (uint32_t y = 1; y + 1 < ny; ++y)
            for (uint32_t x = 1; x + 1 < nx; ++x)
                field[(uint64_t)index(x, y, z)] = FLUID;
    fixOddCells();
}

// Odd cells are 2x2x2 blocks starting at odd indices (xOddStart == false).
// A block lying completely inside the grid that holds a fluid node is made
// entirely fluid.
void LevelGrid::fixOddCells()
{
    auto cellStart = [](int64_t i) { return (i % 2 != 0) ? i : i - 1; };
    for (uint64_t idx = 0; idx < size; ++idx) {
        int64_t ix, iy, iz;
        coords(idx, ix, iy, iz);
        const int64_t x0 = cellStart(ix), y0 = cellStart(iy), z0 = cellStart(iz);
        if (x0 < 0 || y0 < 0 || z0 < 0 || x0 + 1 >= (int64_t)nx || y0 + 1 >= (int64_t)ny || z0 + 1 >= (int64_t)nz)
            continue;
        bool any = false;
        for (int c = 0; c < 8 && !any; ++c)
            any = field[(uint64_t)index(x0 + (c & 1), y0 + ((c >> 1) & 1), z0 + ((c >> 2) & 1))] == FLUID;
        if (any)
            for (int c = 0; c < 8; ++c)
                field[(uint64_t)index(x0 + (c & 1), y0 + ((c >> 1) & 1), z0 + ((c >> 2) & 1))] = FLUID;
    }
}

void LevelGrid::findStoppers()
{
    for (uint64_t idx = 0; idx < size; ++idx) {
        if (field[idx] == INVALID_OUT_OF_GRID && hasNeighborOfType(idx, FLUID))
            field[idx] = level != 0 ? STOPPER_OUT_OF_GRID : STOPPER_OUT_OF_GRID_BOUNDARY;
        if (field[idx] == FLUID && !hasAllNeighbors(idx))
            field[idx] = STOPPER_OUT_OF_GRID_BOUNDARY;
    }
}

// first / last fluid node along an axis through (ix, iy, iz)
// (GridImp::getFirstFluidNode :1182-1193, getLastFluidNode :1170-1180)
int64_t LevelGrid::firstFluidAlong(int64_t ix, int64_t iy, int64_t iz, int axis) const
{
    int64_t c[3] = { ix, iy, iz };
    c[axis] = 0;
    const int64_t n = axis == 0 ? nx : axis == 1 ? ny : nz;
    while (c[axis] < n && !isFluid((uint64_t)index(c[0], c[1], c[2])))
        ++c[axis];
    return c[axis];
}

int64_t LevelGrid::lastFluidAlong(int64_t ix, int64_t iy, int64_t iz, int axis) const
{
    int64_t c[3] = { ix, iy, iz };
    c[axis] = (axis == 0 ? nx : axis == 1 ? ny : nz) - 1;
    while (c[axis] >= 0 && !isFluid((uint64_t)index(c[0], c[1], c[2])))
        --c[axis];
    return c[axis];
}

// GridImp::getNeighborIndex / getPeriodicNeighborCoords (GridImp.cpp:1052-1099)
int64_t LevelGrid::neighborIndexPositive(int64_t ix, int64_t iy, int64_t iz, int axis) const
{
    int64_t c[3] = { ix, iy, iz };
    c[axis] += 1;
    if (periodic[axis]) {
        const int64_t n = index(c[0], c[1], c[2]);
        if (n >= 0 && field[(uint64_t)n] == STOPPER_OUT_OF_GRID_BOUNDARY)
            c[axis] = firstFluidAlong(ix, iy, iz, axis);
    }
    const int64_t m = index(c[0], c[1], c[2]);
    return m < 0 ? -1 : sparseIndex[(uint64_t)m];
}

// GridImp::getNegativeNeighborIndex / getNegativePeriodicNeighborCoords (:1112-1166)
int64_t LevelGrid::negativeNeighborIndex(int64_t ix, int64_t iy, int64_t iz) const
{
    int64_t c[3] = { ix - 1, iy - 1, iz - 1 };
    int64_t self[3] = { ix, iy, iz };
    bool onBoundary[3] = { false, false, false };
    for (int a = 0; a < 3; ++a) {
        if (!periodic[a])
            continue;
        int64_t n[3] = { ix, iy, iz };
        n[a] -= 1;
        // the reference indexes the field with the sparse index of the node
        // (GridImp.cpp:1133-1134); both agree while no node before it was
        // removed from the sparse set
        const int64_t m = index(n[0], n[1], n[2]);
        if (m < 0 || sparseIndex[(uint64_t)m] < 0)
            continue;
        if (field[(uint64_t)sparseIndex[(uint64_t)m]] == STOPPER_OUT_OF_GRID_BOUNDARY)
            onBoundary[a] = true;
    }
    for (int a = 0; a < 3; ++a) {
        if (onBoundary[a]) {
            self[a] = lastFluidAlong(self[0], self[1], self[2], a);
            c[a] = self[a];
        }
    }
    const int64_t m = index(c[0], c[1], c[2]);
    return m < 0 ? -1 : sparseIndex[(uint64_t)m];
}

// GridImp::updateSparseIndices and setNeighborIndices (GridImp.cpp:914-1050)
void LevelGrid::findSparseIndices()
{
    sparseIndex.assign(size, -1);
    int64_t next = 0;
    for (uint64_t i = 0; i < size; ++i) {
        const uint8_t t = field[i];
        if (t == INVALID_COARSE_UNDER_FINE || t == INVALID_OUT_OF_GRID || t == INVALID_SOLID)
            continue;
        sparseIndex[i] = next++;
    }
    sparseSize = (uint64_t)next;

    neighborX.assign(size, -1);
    neighborY.assign(size, -1);
    neighborZ.assign(size, -1);
    neighborNeg.assign(size, -1);
    for (uint64_t i = 0; i < size; ++i) {
        int64_t ix, iy, iz;
        coords(i, ix, iy, iz);
        if (isStopper(i)) {
            // GridImp::setStopperNeighborCoords (:1037-1050)
            auto stopperNeighbor = [&](int64_t jx, int64_t jy, int64_t jz) -> int64_t {
                const int64_t m = index(jx, jy, jz);
                if (m < 0 || field[(uint64_t)m] == INVALID_OUT_OF_GRID)
                    return -1;
                return sparseIndex[(uint64_t)m];
            };
            neighborX[i] = stopperNeighbor(ix + 1, iy, iz);
            neighborY[i] = stopperNeighbor(ix, iy + 1, iz);
            neighborZ[i] = stopperNeighbor(ix, iy, iz + 1);
            continue;
        }
        if (sparseIndex[i] < 0)
            continue;
        neighborX[i] = neighborIndexPositive(ix, iy, iz, 0);
        neighborY[i] = neighborIndexPositive(ix, iy, iz, 1);
        neighborZ[i] = neighborIndexPositive(ix, iy, iz, 2);
        neighborNeg[i] = negativeNeighborIndex(ix, iy, iz);
    }
}

void LevelGrid::findFluidNodes()
{
    fluidNodes.clear();
    for (uint64_t i = 0; i < size; ++i)
        if (sparseIndex[i] >= 0 && isFluid(i))
            fluidNodes.push_back((uint32_t)(sparseIndex[i] + 1));
}

void LevelGrid::nodeValues(std::vector<double>& cxs, std::vector<double>& cys, std::vector<double>& czs,
                           std::vector<uint32_t>& nbx, std::vector<uint32_t>& nby, std::vector<uint32_t>& nbz,
                           std::vector<uint32_t>& nbneg, std::vector<uint32_t>& geo) const
{
    const uint64_t N = sparseSize + 1;
    cxs.assign(N, 0.0);
    cys.assign(N, 0.0);
    czs.assign(N, 0.0);
    nbx.assign(N, 0);
    nby.assign(N, 0);
    nbz.assign(N, 0);
    nbneg.assign(N, 0);
    geo.assign(N, 16);
    geo[0] = 16;
    uint64_t node = 1;
    for (uint64_t i = 0; i < size; ++i) {
        if (sparseIndex[i] < 0)
            continue;
        int64_t ix, iy, iz;
        coords(i, ix, iy, iz);
        cxs[node] = (double)ix * delta + startX;
        cys[node] = (double)iy * delta + startY;
        czs[node] = (double)iz * delta + startZ;
        nbx[node] = (uint32_t)(neighborX[i] + 1);
        nby[node] = (uint32_t)(neighborY[i] + 1);
        nbz[node] = (uint32_t)(neighborZ[i] + 1);
        nbneg[node] = (uint32_t)(neighborNeg[i] + 1);
        geo[node] = isFluid(i) ? 19u : 16u;
        ++node;
    }
}

// q values of one side node (Side::setQs, Side.cpp:149-176), including the
// periodic correction of the neighbour (Side.cpp:222-256), which also moves
// the node's own coordinate used by the diagonal reset that follows.
void LevelGrid::sideQs(SideType side, int64_t ix, int64_t iy, int64_t iz, double* qNode) const
{
    for (int dir = 0; dir < 27; ++dir) {
        int64_t c[3] = { ix, iy, iz };
        int64_t n[3] = { ix + cx(dir), iy + cy(dir), iz + cz(dir) };
        for (int a = 0; a < 3; ++a) {
            if (!periodic[a])
                continue;
            int64_t probe[3] = { c[0], c[1], c[2] };
            probe[a] = n[a];
            const int64_t m = index(probe[0], probe[1], probe[2]);
            if (m < 0 || field[(uint64_t)m] != STOPPER_OUT_OF_GRID_BOUNDARY)
                continue;
            if (n[a] > c[a]) {
                c[a] = firstFluidAlong(c[0], c[1], c[2], a);
                n[a] = c[a];
            } else {
                c[a] = lastFluidAlong(c[0], c[1], c[2], a);
                n[a] = c[a];
            }
        }
        const int64_t nIdx = index(n[0], n[1], n[2]);
        qNode[dir] = (isStopperForBC(nIdx) && alignedWith(dir, side)) ? 0.5 : -1.0;
        // Side::resetDiagonalsInCaseOfOtherBC (Side.cpp:193-215)
        if (qNode[dir] == 0.5) {
            for (SideType other : bcAlreadySet) {
                const int od = sideDirection(other);
                const int64_t m = index(c[0] + cx(od), c[1] + cy(od), c[2] + cz(od));
                if (!isStopperForBC(m))
                    continue;
                if (alignedWith(dir, other))
                    qNode[dir] = -1.0;
            }
        }
    }
}

// ------------------------------------------------------------ GridBuilder --
void GridBuilder::addCoarseGrid(double sx, double sy, double sz, double ex, double ey, double ez, double delta)
{
    // MultipleGridBuilder::addCoarseGrid widens the box by half a spacing
    // (MultipleGridBuilder.cpp:59-72)
    if (!grids.empty())
        throw std::runtime_error("coarse grid already added");
    sx -= 0.5 * delta;
    sy -= 0.5 * delta;
    sz -= 0.5 * delta;
    ex += 0.5 * delta;
    ey += 0.5 * delta;
    ez += 0.5 * delta;
    grids.emplace_back(new LevelGrid(sx, sy, sz, ex, ey, ez, delta, 0));
    velocity.emplace_back();
    slip.emplace_back();
    pressure.emplace_back();
}

void GridBuilder::setPeriodicBoundaryCondition(bool px, bool py, bool pz)
{
    for (auto& g : grids) {
        g->periodic[0] = px;
        g->periodic[1] = py;
        g->periodic[2] = pz;
    }
}

void GridBuilder::buildGrids(bool)
{
    if (grids.empty())
        throw std::runtime_error("buildGrids: no coarse grid");
    for (int level = (int)grids.size() - 1; level >= 0; --level) {
        grids[level]->initialNodes();
        grids[level]->findStoppers();
    }
    for (auto& g : grids) {
        g->findSparseIndices();
        g->findFluidNodes();
    }
    built = true;
}

static void addSide(std::vector<std::unique_ptr<LevelGrid>>& grids, std::vector<std::vector<BCList>>& lists,
                    SideType side, BCKind kind, double v0, double v1, double v2)
{
    for (size_t level = 0; level < grids.size(); ++level) {
        LevelGrid& g = *grids[level];
        const LevelGrid& g0 = *grids[0];
        BCList bc;
        bc.kind = kind;
        bc.side = side;
        bc.d3q27Direction = sideDirection(side);
        const int axis = sideAxis(side);
        const int sgn = sideSign(side);
        const int64_t nAxis = axis == 0 ? g.nx : axis == 1 ? g.ny : g.nz;
        // the first layer inside the stopper layer on this side; finer
        // levels only take part when they reach the coarse side
        // (MX::addIndices etc., Side.cpp:330-404)
        const int64_t layer = sgn < 0 ? 1 : nAxis - 2;
        const double coordNormal = (sgn < 0 ? (axis == 0 ? g.startX : axis == 1 ? g.startY : g.startZ) + g.delta
                                            : (axis == 0 ? g.endX : axis == 1 ? g.endY : g.endZ) - g.delta);
        const double coarseNormal = (sgn < 0 ? (axis == 0 ? g0.startX : axis == 1 ? g0.startY : g0.startZ) + g0.delta
                                             : (axis == 0 ? g0.endX : axis == 1 ? g0.endY : g0.endZ) - g0.delta);
        if ((sgn < 0 && coordNormal > coarseNormal) || (sgn > 0 && coordNormal < coarseNormal)) {
            lists[level].push_back(bc);
            continue;
        }
        const int a1 = axis == 0 ? 1 : 0;      // inner loop axis
        const int a2 = axis == 2 ? 1 : 2;      // outer loop axis
        const int64_t n1 = a1 == 0 ? g.nx : g.ny;
        const int64_t n2 = a2 == 1 ? g.ny : g.nz;
        const uint8_t type = kind == BCKind::Pressure ? BC_PRESSURE : kind == BCKind::Slip ? BC_SLIP : BC_VELOCITY;
        for (int64_t j2 = 0; j2 < n2; ++j2) {
            for (int64_t j1 = 0; j1 < n1; ++j1) {
                int64_t c[3];
                c[axis] = layer;
                c[a1] = j1;
                c[a2] = j2;
                const int64_t idx = g.index(c[0], c[1], c[2]);
                if (idx < 0)
                    continue;
                const uint8_t t = g.field[(uint64_t)idx];
                const bool hasBC =
                    t == BC_PRESSURE || t == BC_VELOCITY || t == BC_NOSLIP || t == BC_SLIP || t == BC_STRESS;
                if (!(t == FLUID || t == FLUID_CFC || t == FLUID_CFF || t == FLUID_FCC || t == FLUID_FCF || hasBC))
                    continue;
                g.field[(uint64_t)idx] = type;
                bc.k.push_back((int32_t)(g.sparseIndex[(uint64_t)idx] + 1));
                if (kind == BCKind::Pressure) {
                    int64_t n[3] = { c[0], c[1], c[2] };
                    n[axis] -= sgn;
                    const int64_t m = g.index(n[0], n[1], n[2]);
                    bc.kN.push_back((int32_t)(g.sparseIndex[(uint64_t)m] + 1));
                    bc.rho.push_back(v0);
                }
                double qNode[27];
                g.sideQs(side, c[0], c[1], c[2], qNode);
                for (int d = 0; d < 27; ++d)
                    bc.q.push_back(qNode[d]);
                if (kind == BCKind::Velocity || kind == BCKind::NoSlip) {
                    bc.vx.push_back(kind == BCKind::NoSlip ? 0.0 : v0);
                    bc.vy.push_back(kind == BCKind::NoSlip ? 0.0 : v1);
                    bc.vz.push_back(kind == BCKind::NoSlip ? 0.0 : v2);
                }
                if (kind == BCKind::Slip) {
                    bc.normalX.push_back(v0);
                    bc.normalY.push_back(v1);
                    bc.normalZ.push_back(v2);
                }
            }
        }
        // node-major q to direction-major
        const size_t n = bc.k.size();
        std::vector<double> q(27 * n);
        for (size_t i = 0; i < n; ++i)
            for (int d = 0; d < 27; ++d)
                q[(size_t)d * n + i] = bc.q[i * 27 + (size_t)d];
        bc.q.swap(q);
        g.bcAlreadySet.push_back(side);
        lists[level].push_back(std::move(bc));
    }
}

void GridBuilder::setNoSlipBoundaryCondition(SideType side)
{
    addSide(grids, velocity, side, BCKind::NoSlip, 0, 0, 0);
}
void GridBuilder::setVelocityBoundaryCondition(SideType side, double vx, double vy, double vz)
{
    addSide(grids, velocity, side, BCKind::Velocity, vx, vy, vz);
}
void GridBuilder::setPressureBoundaryCondition(SideType side, double rho)
{
    addSide(grids, pressure, side, BCKind::Pressure, rho, 0, 0);
}
void GridBuilder::setSlipBoundaryCondition(SideType side, double nx, double ny, double nz)
{
    addSide(grids, slip, side, BCKind::Slip, nx, ny, nz);
}

} // namespace vfb::grid
