// grid_builder.cpp -- see grid_builder.hpp.
#include "grid_builder.hpp"

#include <cfloat>
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

namespace
{
// vf::Math::lessEqual / greaterEqual with the default tolerance
// (utilities/math/Math.cpp:40-64, EPSILON = FLT_EPSILON)
bool nearlyEqual(double a, double b)
{
    const double largest = std::fabs(b) > std::fabs(a) ? std::fabs(b) : std::fabs(a);
    return std::fabs(a - b) <= largest * (double)FLT_EPSILON;
}
bool lessEqualTol(double a, double b) { return a < b || nearlyEqual(a, b); }
bool greaterEqualTol(double a, double b) { return a > b || nearlyEqual(a, b); }
} // namespace

bool Box::containsPoint(double x, double y, double z) const
{
    const double lo[3] = { std::fmin(minX, maxX), std::fmin(minY, maxY), std::fmin(minZ, maxZ) };
    const double hi[3] = { std::fmax(minX, maxX), std::fmax(minY, maxY), std::fmax(minZ, maxZ) };
    const double p[3] = { x, y, z };
    for (int a = 0; a < 3; ++a)
        if (lessEqualTol(p[a], lo[a]) || greaterEqualTol(p[a], hi[a]))
            return false;
    return true;
}

bool Solid::contains(double x, double y, double z) const
{
    if (kind == Kind::Cuboid)
        return box.containsPoint(x, y, z);
    if (kind == Kind::Conglomerate) {
        // Conglomerate::isPointInObject (Conglomerate.cpp:153-164)
        for (const Solid& part : subtract)
            if (part.contains(x, y, z))
                return false;
        for (const Solid& part : add)
            if (part.contains(x, y, z))
                return true;
        return false;
    }
    if (kind == Kind::Cylinder) {
        // Cylinder::isPointInObject with zero offsets (Cylinder.cpp:163-187):
        // within half the height along the axis, strictly inside the circle
        const double d[3] = { x - cx, y - cy, z - cz };
        const double along = d[axis];
        if (along > 0.5 * height || along < -0.5 * height)
            return false;
        const double a = d[(axis + 1) % 3], b = d[(axis + 2) % 3];
        const double u = axis == 1 ? b : a, v = axis == 1 ? a : b; // the reference's (x, z) order for the y axis
        return (u * u + v * v) < (r * r);
    }
    // Sphere::isPointInObject with zero offsets (Sphere.cpp)
    const double dx = x - cx, dy = y - cy, dz = z - cz;
    return (dx * dx + dy * dy + dz * dz) < (r * r);
}

// Sphere::getIntersection (Sphere.cpp): the roots of |p + t d - c|^2 = r^2,
// the smaller non-negative one
bool Solid::intersect(double px, double py, double pz, double dx, double dy, double dz, double& t) const
{
    if (kind != Kind::Sphere) // Object::getIntersection (Object.cpp:42-45) reports no hit
        return false;
    const double rx = px - cx, ry = py - cy, rz = pz - cz;
    const double dd = dx * dx + dy * dy + dz * dz;
    const double p = 2 * (rx * dx + ry * dy + rz * dz) / dd;
    const double q = (rx * rx + ry * ry + rz * rz - r * r) / dd;
    const double disc = 0.25 * p * p - q;
    if (disc < 0.0)
        return false;
    double t1 = -0.5 * p + std::sqrt(disc);
    double t2 = -0.5 * p - std::sqrt(disc);
    if (t1 < 0.0 && t2 < 0.0)
        return false;
    if (t1 < 0.0)
        t1 = (double)FLT_MAX;
    if (t2 < 0.0)
        t2 = (double)FLT_MAX;
    t = t2 < t1 ? t2 : t1;
    return true;
}

int64_t LevelGrid::coordToIndex(double x, double y, double z) const
{
    const long ix = std::lround((x - startX) / delta);
    const long iy = std::lround((y - startY) / delta);
    const long iz = std::lround((z - startZ) / delta);
    if (ix < 0 || iy < 0 || iz < 0 || ix >= (long)nx || iy >= (long)ny || iz >= (long)nz)
        return -1;
    return (int64_t)ix + (int64_t)nx * ((int64_t)iy + (int64_t)ny * (int64_t)iz);
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

// The node types of one level (GridImp::inital, GridImp.cpp:122-194): the
// inner region (the coarse level: everything but the outermost layer,
// GridImp::findInnerNode :228-248; a refined level: the nodes whose odd cell
// lies inside the refinement box; an intermediate level: the nodes with a
// fluid child on the finer level, :311-336), the overlap layers (:338-366),
// the completed odd cells (:465-472) and the end-of-grid stoppers (:436-448).
void LevelGrid::initial(const LevelGrid* finer)
{
    field.assign(size, INVALID_OUT_OF_GRID);
    if (innerFromFiner) {
        if (!finer)
            throw std::runtime_error("intermediate level without a finer level");
        setInnerBasedOnFinerGrid(*finer);
    } else {
        findInnerNodes();
    }
    addOverlap();
    fixOddCells();
    findStoppers();
}

// start index of the odd cell (2x2x2 block) holding index i along an axis
// (GridImp::getOddCellFromIndex, GridImp.cpp:287-309)
int64_t LevelGrid::oddCellStart(int64_t i, int axis) const
{
    const bool odd = (i % 2) != 0;
    return oddStart[axis] ? (odd ? i - 1 : i) : (odd ? i : i - 1);
}

void LevelGrid::findInnerNodes()
{
    if (level == 0) {
        for (uint32_t z = 1; z + 1 < nz; ++z)
            for (uint32_t y = 1; y + 1 < ny; ++y)
                for (uint32_t x = 1; x + 1 < nx; ++x)
                    field[(uint64_t)index(x, y, z)] = FLUID;
        return;
    }
    if (!hasShape)
        throw std::runtime_error("refined level without a refinement box");
    for (uint64_t idx = 0; idx < size; ++idx) {
        int64_t ix, iy, iz;
        coords(idx, ix, iy, iz);
        // the cell's corner coordinates as the reference forms them: the
        // node's coordinate, or one spacing below it, plus 0 / 1 spacing
        const double x = coordX(ix), y = coordY(iy), z = coordZ(iz);
        const double xs = oddCellStart(ix, 0) == ix ? x : x - delta;
        const double ys = oddCellStart(iy, 1) == iy ? y : y - delta;
        const double zs = oddCellStart(iz, 2) == iz ? z : z - delta;
        bool inside = true;
        for (int c = 0; c < 8 && inside; ++c)
            inside = shape.containsPoint((c & 1) ? xs + delta : xs, (c & 2) ? ys + delta : ys,
                                         (c & 4) ? zs + delta : zs);
        if (inside)
            field[idx] = FLUID;
    }
}

void LevelGrid::setInnerBasedOnFinerGrid(const LevelGrid& fine)
{
    for (uint64_t idx = 0; idx < size; ++idx) {
        int64_t ix, iy, iz;
        coords(idx, ix, iy, iz);
        const double x = coordX(ix), y = coordY(iy), z = coordZ(iz);
        const double q = 0.25 * delta;
        // children in the order of GridImp.cpp:318-325 (+ before -, z fastest)
        for (int c = 0; c < 8; ++c) {
            const double cxq = (c & 4) ? x - q : x + q;
            const double cyq = (c & 2) ? y - q : y + q;
            const double czq = (c & 1) ? z - q : z + q;
            const int64_t child = fine.coordToIndex(cxq, cyq, czq);
            if (child >= 0 && fine.field[(uint64_t)child] == FLUID) {
                field[idx] = FLUID;
                break;
            }
        }
    }
}

void LevelGrid::addOverlap()
{
    for (uint32_t layer = 0; layer < numberOfLayers; ++layer) {
        for (uint64_t idx = 0; idx < size; ++idx)
            if (field[idx] == INVALID_OUT_OF_GRID && hasNeighborOfType(idx, FLUID))
                field[idx] = OVERLAP_TMP;
        for (uint64_t idx = 0; idx < size; ++idx)
            if (field[idx] == OVERLAP_TMP)
                field[idx] = FLUID;
    }
}

// A 2x2x2 odd cell lying completely inside the grid that holds a fluid node
// is made entirely fluid.  Odd cells tile the grid, so the result does not
// depend on the visiting order.
void LevelGrid::fixOddCells()
{
    for (uint64_t idx = 0; idx < size; ++idx) {
        int64_t ix, iy, iz;
        coords(idx, ix, iy, iz);
        const int64_t x0 = oddCellStart(ix, 0), y0 = oddCellStart(iy, 1), z0 = oddCellStart(iz, 2);
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

// ------------------------------------------------------------------ solid --
// GridImp::mesh for a geometric primitive (GridImp.cpp:1300-1320): nodes
// strictly inside the cuboid become INVALID_SOLID (GridImp::discretize
// :251-268), needle cells are closed (:1362-1401), INVALID_SOLID nodes next to
// fluid become STOPPER_SOLID (:449-453) and fluid nodes next to those BC_SOLID,
// numbered in matrix order (:455-463).  With thin walls
// (MultipleGridBuilder.cpp:543-552) BC_SOLID nodes without a fluid neighbour
// become STOPPER_SOLID before the q computation (GridImp::closeNeedleCellsThinWall,
// GridImp.cpp:1403-1434); they keep their q slot, which stays unused.  The
// reference's preceding search for further boundary nodes
// (findQsPrimitive in the FindSolidBoundaryNodes stage, :1522-1555) only
// visits nodes that already have a q slot, which are BC_SOLID, never FLUID,
// so for a primitive it changes nothing and is not repeated here.
void LevelGrid::meshSolid(const Solid& solid, bool thinWalls)
{
    for (uint64_t idx = 0; idx < size; ++idx) {
        if (field[idx] == INVALID_SOLID)
            continue;
        int64_t ix, iy, iz;
        coords(idx, ix, iy, iz);
        if (solid.contains(coordX(ix), coordY(iy), coordZ(iz)))
            field[idx] = INVALID_SOLID;
    }
    auto isSolidAt = [&](int64_t jx, int64_t jy, int64_t jz) {
        const int64_t m = index(jx, jy, jz);
        return m >= 0 && field[(uint64_t)m] == INVALID_SOLID;
    };
    uint64_t closed;
    do {
        closed = 0;
        for (uint64_t idx = 0; idx < size; ++idx) {
            if (field[idx] != FLUID)
                continue;
            int64_t ix, iy, iz;
            coords(idx, ix, iy, iz);
            if ((isSolidAt(ix + 1, iy, iz) && isSolidAt(ix - 1, iy, iz)) ||
                (isSolidAt(ix, iy + 1, iz) && isSolidAt(ix, iy - 1, iz)) ||
                (isSolidAt(ix, iy, iz + 1) && isSolidAt(ix, iy, iz - 1))) {
                field[idx] = INVALID_SOLID;
                ++closed;
            }
        }
    } while (closed > 0);
    for (uint64_t idx = 0; idx < size; ++idx)
        if (field[idx] == INVALID_SOLID && hasNeighborOfType(idx, FLUID))
            field[idx] = STOPPER_SOLID;
    solidBoundaryIndex.assign(size, -1);
    numberOfSolidBoundaryNodes = 0;
    for (uint64_t idx = 0; idx < size; ++idx) {
        if (field[idx] == FLUID && hasNeighborOfType(idx, STOPPER_SOLID)) {
            field[idx] = BC_SOLID;
            solidBoundaryIndex[idx] = numberOfSolidBoundaryNodes++;
        }
    }
    if (thinWalls) {
        // closing a node changes no FLUID node, so one pass reaches the fixed point
        for (uint64_t idx = 0; idx < size; ++idx)
            if (field[idx] == BC_SOLID && !hasNeighborOfType(idx, FLUID))
                field[idx] = STOPPER_SOLID;
    }
    // GridImp::findQsPrimitive / calculateQs (GridImp.cpp:1522-1596): per
    // BC_SOLID node and link to a node of the grid, the distance to the
    // surface along the link in lattice spacings, kept when it lies in
    // [0, 1] (with the reference's relative tolerance).  The rest direction
    // has no length and never yields a value.
    const uint32_t nS = numberOfSolidBoundaryNodes;
    solidQ.assign(27 * (size_t)nS, -1.0);
    for (uint64_t idx = 0; idx < size; ++idx) {
        if (field[idx] != BC_SOLID)
            continue;
        int64_t ix, iy, iz;
        coords(idx, ix, iy, iz);
        const double x = coordX(ix), y = coordY(iy), z = coordZ(iz);
        for (int d = 1; d < 27; ++d) {
            const double dx = (double)vfb::cx(d), dy = (double)vfb::cy(d), dz = (double)vfb::cz(d);
            if (coordToIndex(x + dx * delta, y + dy * delta, z + dz * delta) < 0)
                continue;
            double t;
            if (!solid.intersect(x, y, z, dx, dy, dz, t))
                continue;
            const double sub = t / delta;
            double& qv = solidQ[(size_t)d * nS + (size_t)solidBoundaryIndex[idx]];
            if (lessEqualTol(sub, 1.0) && greaterEqualTol(sub, 0.0) && (-0.5 > qv || sub < qv))
                qv = sub;
        }
    }
}

// Geometry::addIndices (Side.cpp:270-307): the links' q values (a cuboid has
// no ray intersection, Object::getIntersection, so all its q stay -1), and a
// link without one gets q = 1/2 when its neighbour is a stopper node.
void LevelGrid::geometryList(std::vector<int32_t>& k, std::vector<double>& q) const
{
    std::vector<int64_t> nodes;
    for (uint64_t idx = 0; idx < size; ++idx)
        if (field[idx] == BC_SOLID)
            nodes.push_back((int64_t)idx);
    const size_t n = nodes.size();
    k.assign(n, 0);
    q.assign(27 * n, -1.0);
    for (size_t i = 0; i < n; ++i) {
        const uint64_t idx = (uint64_t)nodes[i];
        k[i] = (int32_t)(sparseIndex[idx] + 1);
        int64_t ix, iy, iz;
        coords(idx, ix, iy, iz);
        for (int d = 0; d < 27; ++d) {
            double qd = solidQ[(size_t)d * numberOfSolidBoundaryNodes + (size_t)solidBoundaryIndex[idx]];
            const int64_t m = index(ix + cx(d), iy + cy(d), iz + cz(d));
            if (qd < -0.5 && m >= 0) {
                const uint8_t t = field[(uint64_t)m];
                if (t == STOPPER_OUT_OF_GRID_BOUNDARY || t == STOPPER_OUT_OF_GRID || t == STOPPER_SOLID)
                    qd = 0.5;
            }
            q[(size_t)d * n + i] = qd;
        }
    }
}

// -------------------------------------------------------------- interface --
// (GridInterface.cpp).  Coordinates are mapped between the levels with the
// reference's own arithmetic: a coarse node and the fine node a quarter coarse
// spacing above / below it.
int64_t LevelGrid::coarseToFineIndex(uint64_t idx, const LevelGrid& fine) const
{
    int64_t ix, iy, iz;
    coords(idx, ix, iy, iz);
    return fine.coordToIndex(coordX(ix) + fine.delta * 0.5, coordY(iy) + fine.delta * 0.5, coordZ(iz) + fine.delta * 0.5);
}

int64_t LevelGrid::fineToCoarseIndex(uint64_t idx, const LevelGrid& fine) const
{
    int64_t ix, iy, iz;
    coords(idx, ix, iy, iz);
    return fine.coordToIndex(coordX(ix) - fine.delta * 0.5, coordY(iy) - fine.delta * 0.5, coordZ(iz) - fine.delta * 0.5);
}

// GridInterface::isNeighborFineInvalid (:254-271)
bool LevelGrid::isNeighborFineInvalid(int64_t jx, int64_t jy, int64_t jz, const LevelGrid& fine) const
{
    const int64_t nb = index(jx, jy, jz);
    if (nb < 0)
        return false;
    const uint8_t t = field[(uint64_t)nb];
    if (t == STOPPER_OUT_OF_GRID || t == STOPPER_OUT_OF_GRID_BOUNDARY)
        return false;
    const int64_t f = coarseToFineIndex((uint64_t)nb, fine);
    if (f < 0)
        return true;
    const uint8_t ft = fine.field[(uint64_t)f];
    return ft == INVALID_OUT_OF_GRID || ft == STOPPER_OUT_OF_GRID;
}

// the cell starting at (x0, y0, z0) lies in the grid and holds only types a / b
bool LevelGrid::cellContainsOnly(int64_t x0, int64_t y0, int64_t z0, uint8_t a, uint8_t b) const
{
    for (int c = 0; c < 8; ++c) {
        const int64_t m = index(x0 + (c & 1), y0 + ((c >> 1) & 1), z0 + ((c >> 2) & 1));
        if (m < 0)
            return false;
        const uint8_t t = field[(uint64_t)m];
        if (t != a && t != b)
            return false;
    }
    return true;
}

// GridImp::setNonStopperOutOfGridCellTo (:708-724): the cell starting at the node
void LevelGrid::setNonStopperOutOfGridCellTo(uint64_t idx, uint8_t type)
{
    int64_t ix, iy, iz;
    coords(idx, ix, iy, iz);
    for (int c = 0; c < 8; ++c) {
        const int64_t m = index(ix + (c & 1), iy + ((c >> 1) & 1), iz + ((c >> 2) & 1));
        if (m < 0)
            continue;
        const uint8_t t = field[(uint64_t)m];
        if (t != STOPPER_OUT_OF_GRID && t != STOPPER_OUT_OF_GRID_BOUNDARY)
            field[(uint64_t)m] = type;
    }
}

// GridInterface::findOffsetCF (:372-399): the node's own cell if it holds
// only fluid / coarse-to-fine nodes, else the first neighbour cell (in
// direction order) that does; offset = that direction
int64_t LevelGrid::offsetCellCF(uint64_t idx, int& offset) const
{
    int64_t ix, iy, iz;
    coords(idx, ix, iy, iz);
    offset = d000;
    if (cellContainsOnly(ix, iy, iz, FLUID, FLUID_CFC))
        return (int64_t)idx;
    for (int d = 0; d < 27; ++d) {
        if (cellContainsOnly(ix + cx(d), iy + cy(d), iz + cz(d), FLUID, FLUID_CFC)) {
            offset = d;
            return index(ix + cx(d), iy + cy(d), iz + cz(d));
        }
    }
    return (int64_t)idx;
}

// GridInterface::findOffsetFC (:401-428), on the fine level.  The neighbour
// cells are tested for fluid / coarse-to-fine types, as the reference does.
int64_t LevelGrid::offsetCellFC(uint64_t idx, int& offset) const
{
    int64_t ix, iy, iz;
    coords(idx, ix, iy, iz);
    offset = d000;
    if (cellContainsOnly(ix, iy, iz, FLUID, FLUID_FCF))
        return (int64_t)idx;
    for (int d = 0; d < 27; ++d) {
        if (cellContainsOnly(ix + cx(d), iy + cy(d), iz + cz(d), FLUID, FLUID_CFC)) {
            offset = d;
            return index(ix + cx(d), iy + cy(d), iz + cz(d));
        }
    }
    return (int64_t)idx;
}

// GridImp::findGridInterface (:1204-1232): coarse-to-fine cells (fluid and
// boundary-stopper variants, GridInterface.cpp:60-122), then fine-to-coarse
// cells (:125-158), then the coarse nodes under the fine level (:160-196),
// each a pass over the coarse level in matrix order.
void LevelGrid::findGridInterface(LevelGrid& fine)
{
    cf = InterfaceCells();
    fc = InterfaceCells();
    auto addCF = [&](uint64_t idx, int64_t f) {
        int64_t ix, iy, iz;
        coords(idx, ix, iy, iz);
        for (int d = 0; d < 27; ++d) {
            if (isNeighborFineInvalid(ix + cx(d), iy + cy(d), iz + cz(d), fine)) {
                int offset;
                const int64_t c = offsetCellCF(idx, offset);
                cf.coarse.push_back(c);
                cf.fine.push_back(f);
                cf.offset.push_back(offset);
                setNonStopperOutOfGridCellTo(idx, FLUID_CFC);
                fine.setNonStopperOutOfGridCellTo((uint64_t)f, FLUID_CFF);
                return;
            }
        }
    };
    for (uint64_t idx = 0; idx < size; ++idx) {
        if (isFluid(idx)) {
            const int64_t f = coarseToFineIndex(idx, fine);
            if (f >= 0 && fine.isFluid((uint64_t)f))
                addCF(idx, f);
        }
        if (field[idx] == STOPPER_OUT_OF_GRID_BOUNDARY) {
            const int64_t f = coarseToFineIndex(idx, fine);
            if (f >= 0 && fine.field[(uint64_t)f] == STOPPER_OUT_OF_GRID_BOUNDARY)
                addCF(idx, f);
        }
    }
    for (uint64_t idx = 0; idx < size; ++idx) {
        if (!isFluid(idx) || field[idx] == FLUID_CFC)
            continue;
        const int64_t f = fineToCoarseIndex(idx, fine);
        if (f < 0 || !fine.isFluid((uint64_t)f))
            continue;
        int64_t ix, iy, iz;
        coords(idx, ix, iy, iz);
        for (int d = 0; d < 27; ++d) {
            const int64_t nb = index(ix + cx(d), iy + cy(d), iz + cz(d));
            if (nb >= 0 && field[(uint64_t)nb] == FLUID_CFC) {
                int offset;
                const int64_t fcell = fine.offsetCellFC((uint64_t)f, offset);
                fc.coarse.push_back((int64_t)idx);
                fc.fine.push_back(fcell);
                fc.offset.push_back(offset);
                fine.setNonStopperOutOfGridCellTo((uint64_t)f, FLUID_FCF);
                field[idx] = FLUID_FCC;
                break;
            }
        }
    }
    for (uint64_t idx = 0; idx < size; ++idx) {
        if (!isFluid(idx) || field[idx] == FLUID_CFC || field[idx] == FLUID_FCC)
            continue;
        const int64_t f = fineToCoarseIndex(idx, fine);
        if (f < 0)
            continue;
        if (hasNeighborOfType(idx, FLUID_FCC)) {
            field[idx] = STOPPER_COARSE_UNDER_FINE;
            continue;
        }
        const uint8_t ft = fine.field[(uint64_t)f];
        if (ft == INVALID_SOLID || fine.isFluid((uint64_t)f) || ft == STOPPER_SOLID || ft == BC_SOLID)
            field[idx] = INVALID_COARSE_UNDER_FINE;
    }
}

// GridInterface::repairGridInterfaceOnMultiGPU (:298-361): keep the
// coarse-to-fine cells whose coarse cell holds only coarse-to-fine nodes and
// the fine-to-coarse cells whose fine cell holds only fine-to-coarse nodes
void LevelGrid::repairGridInterface(const LevelGrid& fine)
{
    InterfaceCells keepCF, keepFC;
    for (size_t i = 0; i < cf.size(); ++i) {
        int64_t ix, iy, iz;
        coords((uint64_t)cf.coarse[i], ix, iy, iz);
        if (cellContainsOnly(ix, iy, iz, FLUID_CFC, FLUID_CFC)) {
            keepCF.coarse.push_back(cf.coarse[i]);
            keepCF.fine.push_back(cf.fine[i]);
            keepCF.offset.push_back(cf.offset[i]);
        }
    }
    for (size_t i = 0; i < fc.size(); ++i) {
        int64_t ix, iy, iz;
        fine.coords((uint64_t)fc.fine[i], ix, iy, iz);
        if (fine.cellContainsOnly(ix, iy, iz, FLUID_FCF, FLUID_FCF)) {
            keepFC.coarse.push_back(fc.coarse[i]);
            keepFC.fine.push_back(fc.fine[i]);
            keepFC.offset.push_back(fc.offset[i]);
        }
    }
    cf = std::move(keepCF);
    fc = std::move(keepFC);
}

// GridInterface::findSparseIndex (:363-369): matrix to sparse indices (both
// levels' sparse indices must be current)
void LevelGrid::renumberGridInterface(const LevelGrid& fine)
{
    for (size_t i = 0; i < cf.size(); ++i) {
        cf.coarse[i] = sparseIndex[(uint64_t)cf.coarse[i]];
        cf.fine[i] = fine.sparseIndex[(uint64_t)cf.fine[i]];
    }
    for (size_t i = 0; i < fc.size(); ++i) {
        fc.coarse[i] = sparseIndex[(uint64_t)fc.coarse[i]];
        fc.fine[i] = fine.sparseIndex[(uint64_t)fc.fine[i]];
    }
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
    stress.emplace_back();
    pressure.emplace_back();
}

void GridBuilder::setNumberOfLayers(uint32_t fine, uint32_t betweenLevels)
{
    layersFine = fine;
    layersBetweenLevels = betweenLevels;
}

// MultipleGridBuilder::getStaggeredCoordinates (MultipleGridBuilder.cpp:228-356),
// step for step in the same floating-point operations: the box widened by
// the overlap of this level, snapped to the parent's nodes, staggered by a
// quarter parent spacing, grown by one parent spacing until it covers the
// box, and pulled back inside the parent (odd start) where it sticks out.
std::array<double, 6> GridBuilder::staggeredCoordinates(const Box& shape, int level, int levelFine, bool odd[3]) const
{
    const LevelGrid& parent = *grids[(size_t)level - 1];
    const double deltaCoarse = parent.delta;
    const double delta = 0.5 * deltaCoarse;
    double lo[3] = { std::fmin(shape.minX, shape.maxX), std::fmin(shape.minY, shape.maxY),
                     std::fmin(shape.minZ, shape.maxZ) };
    double hi[3] = { std::fmax(shape.minX, shape.maxX), std::fmax(shape.minY, shape.maxY),
                     std::fmax(shape.minZ, shape.maxZ) };
    if (levelFine >= level) {
        double overlap = 0.0;
        if (level != levelFine) {
            overlap += (double)(layersBetweenLevels + 1) * delta;
            overlap *= 2.0 * (1.0 - std::pow(0.5, (double)(unsigned)(levelFine - level)));
        }
        overlap += (double)layersFine * delta * std::pow(0.5, (double)(unsigned)(levelFine - level));
        for (int a = 0; a < 3; ++a) {
            lo[a] -= overlap;
            hi[a] += overlap;
        }
    }
    const double pStart[3] = { parent.startX, parent.startY, parent.startZ };
    const double pEnd[3] = { parent.endX, parent.endY, parent.endZ };
    std::array<double, 6> c { pStart[0], pStart[1], pStart[2], pEnd[0], pEnd[1], pEnd[2] };
    for (int a = 0; a < 3; ++a)
        while (c[a] < lo[a])
            c[a] += deltaCoarse;
    for (int a = 0; a < 3; ++a)
        while (c[3 + a] > hi[a])
            c[3 + a] -= deltaCoarse;
    for (int a = 0; a < 3; ++a) {
        c[a] -= 0.25 * deltaCoarse;
        c[3 + a] += 0.25 * deltaCoarse;
    }
    for (int a = 0; a < 3; ++a)
        if (c[a] > lo[a])
            c[a] -= deltaCoarse;
    for (int a = 0; a < 3; ++a)
        if (c[3 + a] < hi[a])
            c[3 + a] += deltaCoarse;
    for (int a = 0; a < 3; ++a)
        odd[a] = c[a] < pStart[a];
    for (int a = 0; a < 3; ++a)
        while (c[a] < pStart[a])
            c[a] += delta;
    for (int a = 0; a < 3; ++a)
        while (c[3 + a] > pEnd[a])
            c[3 + a] -= delta;
    return c;
}

void GridBuilder::addGrid(const Box& box, int levelFine)
{
    if (grids.empty())
        throw std::runtime_error("addGrid: add the coarse grid first");
    if (built)
        throw std::runtime_error("addGrid after buildGrids");
    if (levelFine < (int)grids.size())
        throw std::runtime_error("addGrid: level already exists");
    for (int level = (int)grids.size(); level <= levelFine; ++level) {
        bool odd[3];
        const std::array<double, 6> c = staggeredCoordinates(box, level, levelFine, odd);
        double delta = grids[0]->delta; // MultipleGridBuilder::calculateDelta
        for (int i = 0; i < level; ++i)
            delta *= 0.5;
        auto* g = new LevelGrid(c[0], c[1], c[2], c[3], c[4], c[5], delta, level);
        for (int a = 0; a < 3; ++a) {
            g->oddStart[a] = odd[a];
            g->periodic[a] = false;
        }
        g->hasShape = true;
        g->shape = box;
        g->innerFromFiner = level != levelFine;
        g->numberOfLayers = level != levelFine ? layersBetweenLevels : layersFine;
        grids.emplace_back(g);
        velocity.emplace_back();
        slip.emplace_back();
        stress.emplace_back();
        pressure.emplace_back();
    }
}

void GridBuilder::addGeometry(const Solid& s)
{
    if (built)
        throw std::runtime_error("addGeometry after buildGrids");
    hasSolid = true;
    solid = s;
}

void GridBuilder::setPeriodicBoundaryCondition(bool px, bool py, bool pz)
{
    for (auto& g : grids) {
        g->periodic[0] = px;
        g->periodic[1] = py;
        g->periodic[2] = pz;
    }
}

// MultipleGridBuilder::buildGrids (MultipleGridBuilder.cpp:469-597): levels
// initialised from the finest to the coarsest, the solid on the finest
// level, the interfaces between neighbouring levels, their repair, then the
// sparse renumbering (interface cells included).
void GridBuilder::buildGrids(bool enableThinWalls)
{
    if (grids.empty())
        throw std::runtime_error("buildGrids: no coarse grid");
    const int L = (int)grids.size();
    for (int level = L - 1; level >= 0; --level)
        grids[level]->initial(level + 1 < L ? grids[level + 1].get() : nullptr);
    if (hasSolid)
        grids[L - 1]->meshSolid(solid, enableThinWalls);
    for (int level = 0; level + 1 < L; ++level)
        grids[level]->findGridInterface(*grids[level + 1]);
    for (int level = 0; level + 1 < L; ++level)
        grids[level]->repairGridInterface(*grids[level + 1]);
    for (int level = 0; level < L; ++level)
        grids[level]->findSparseIndices();
    for (int level = 0; level + 1 < L; ++level)
        grids[level]->renumberGridInterface(*grids[level + 1]);
    for (auto& g : grids)
        g->findFluidNodes();
    built = true;
}

void GridBuilder::setNoSlipGeometryBoundaryCondition()
{
    if (!built)
        throw std::runtime_error("boundary conditions need buildGrids first");
    if (!hasSolid)
        throw std::runtime_error("no geometry was added");
    geometryNoSlip = true;
}

// LevelGridBuilder::setVelocityGeometryBoundaryCondition (LevelGridBuilder.cpp:176-194):
// the geometry list with one velocity for all its nodes
void GridBuilder::setVelocityGeometryBoundaryCondition(double vx, double vy, double vz)
{
    setNoSlipGeometryBoundaryCondition();
    geometryHasValues = true;
    geometryValues = { vx, vy, vz };
}

// stress sides: the sampling offset (nodes) and the level-0 roughness length and spacing
struct StressParams {
    uint32_t samplingOffset = 0;
    double z0 = 0, dx = 1;
};

static void addSide(std::vector<std::unique_ptr<LevelGrid>>& grids, std::vector<std::vector<BCList>>& lists,
                    SideType side, BCKind kind, double v0, double v1, double v2, const StressParams& sp = {})
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
        const uint8_t type = kind == BCKind::Pressure ? BC_PRESSURE
                             : kind == BCKind::Slip   ? BC_SLIP
                             : kind == BCKind::Stress ? BC_STRESS
                                                      : BC_VELOCITY;
        // StressBoundaryCondition::make(..., z0 * pow(2.0f, level) / dx) (LevelGridBuilder.cpp:135)
        const double z0Level = sp.z0 * std::ldexp(1.0, (int)level) / sp.dx;
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
                if (kind == BCKind::Slip || kind == BCKind::Stress) {
                    bc.normalX.push_back(v0);
                    bc.normalY.push_back(v1);
                    bc.normalZ.push_back(v2);
                }
                if (kind == BCKind::Stress) {
                    // Side::setStressSamplingIndices (Side.cpp:125-145): samplingOffset
                    // nodes from the BC node against the side's outward direction
                    int64_t m[3] = { c[0], c[1], c[2] };
                    m[axis] -= (int64_t)sgn * (int64_t)sp.samplingOffset;
                    const int64_t at = g.index(m[0], m[1], m[2]);
                    if (at < 0 || g.sparseIndex[(uint64_t)at] < 0)
                        throw std::invalid_argument("the stress BC's sampling node lies outside the grid");
                    bc.kN.push_back((int32_t)(g.sparseIndex[(uint64_t)at] + 1));
                    bc.samplingOffset.push_back((int32_t)sp.samplingOffset);
                    bc.z0.push_back(z0Level);
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
void GridBuilder::setStressBoundaryCondition(SideType side, double nx, double ny, double nz, uint32_t samplingOffset,
                                             double z0, double dx)
{
    if (!(dx > 0) || !(z0 > 0))
        throw std::invalid_argument("the stress BC needs z0 > 0 and dx > 0");
    addSide(grids, stress, side, BCKind::Stress, nx, ny, nz, StressParams { samplingOffset, z0, dx });
}

} // namespace vfb::grid
