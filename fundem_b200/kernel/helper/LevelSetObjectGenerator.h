// LevelSetObject:: -- shapes, surface meshes and signed-distance grids for
// level-set particles and walls, with the class names, methods and argument
// meaning of the reference's kernel/helper/LevelSetObjectGenerator.h, so that
// apps written against it compile unchanged.
//
// What differs is where the grid is evaluated.  The reference fills the grid
// on the host, one virtual call per node (Base::buildGrid, :122-224).  Here
// the built-in shapes describe themselves to fundem_levelset_grid, which
// evaluates every node on the GPU in one launch; only a class derived by the
// user (with its own implicit function) is evaluated on the host through the
// virtual function, as in the reference.
//
// The surface meshes (the particles' boundary nodes) are built on the host in
// the reference's vertex order, because contact lists are numbered by node:
// the golden-ratio icosahedron, the midpoint subdivision that numbers new
// vertices by first use of each edge, the cylinder rings and the box corners.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <fstream>
#include <iostream>
#include <limits>
#include <stdexcept>
#include <string>
#include <typeinfo>
#include <unordered_map>
#include <utility>
#include <vector>

#include "../CUDAKernelFunction/myUtility/myVec.h"
#include "fundem_b200.h"

namespace LevelSetObject
{

namespace Utility
{
// |value|^exponent (LevelSetObjectGenerator.h:23-27)
inline double safeAbsPow(const double value, const double exponent) { return std::pow(std::fabs(value), exponent); }
inline double signNoZero(const double value) { return value >= 0.0 ? 1.0 : -1.0; }
inline double clampValue(const double value, const double lowerBound, const double upperBound)
{
    return std::max(lowerBound, std::min(value, upperBound));
}
// walls are positive inside: value and gradient change sign (:41-50)
inline void applyLevelSetSign(double& value, double3& gradient, const bool levelSetPositiveInside)
{
    if (!levelSetPositiveInside) return;
    value = -value;
    gradient = -gradient;
}
}  // namespace Utility

// grid of signed distances: negative inside, positive outside, x fastest (:56-70)
class GridInfo
{
public:
    double3 gridOrigin{0.0, 0.0, 0.0};
    int3 gridNodeSize{0, 0, 0};
    double gridNodeSpacing{0.0};
    std::vector<double> gridNodeSignedDistance;
};

class Base
{
protected:
    GridInfo gridInfo_;

    // A shape the GPU can evaluate fills `shape` and returns true.  Each
    // built-in class answers only for its own exact type, so a user class that
    // overrides the implicit function is evaluated on the host instead.
    virtual bool describeShape(fundem_shape& shape) const
    {
        (void)shape;
        return false;
    }

public:
    Base() = default;
    virtual ~Base() = default;
    Base(const Base&) = default;
    Base(Base&&) noexcept = default;
    Base& operator=(const Base&) = default;
    Base& operator=(Base&&) noexcept = default;

    void clearGrid() { gridInfo_ = GridInfo{}; }
    bool isGridBuilt() const { return !gridInfo_.gridNodeSignedDistance.empty(); }

    virtual bool isValid() const = 0;
    virtual void evaluateImplicitFunctionValueAndGradient(double& implicitFunctionValue,
                                                          double3& implicitFunctionGradient,
                                                          const double3& point) const = 0;
    virtual double3 boundingBoxMin() const = 0;
    virtual double3 boundingBoxMax() const = 0;

    // Base::buildGrid (:122-224): the bounding box padded by max(1, layers)
    // spacings, snapped outwards to multiples of the spacing; each node holds
    // f / |grad f|, or +-spacing/2 where |grad f| <= 1e-12.
    void buildGrid(const double backgroundGridNodeSpacing, const int backgroundGridPaddingLayers = 2)
    {
        clearGrid();
        if (!isValid() || backgroundGridNodeSpacing <= 0.0) return;
        const double h = backgroundGridNodeSpacing;
        const double pad = double(std::max(1, backgroundGridPaddingLayers)) * h;
        const double3 bmin = boundingBoxMin();
        const double3 bmax = boundingBoxMax();
        const double lo[3] = {h * std::floor((bmin.x - pad) / h), h * std::floor((bmin.y - pad) / h),
                              h * std::floor((bmin.z - pad) / h)};
        const double hi[3] = {h * std::ceil((bmax.x + pad) / h), h * std::ceil((bmax.y + pad) / h),
                              h * std::ceil((bmax.z + pad) / h)};
        int n[3];
        for (int a = 0; a < 3; ++a) n[a] = int(std::floor((hi[a] - lo[a]) / h + 0.5)) + 1;
        if (n[0] <= 0 || n[1] <= 0 || n[2] <= 0) return;
        GridInfo g;
        g.gridNodeSpacing = h;
        g.gridOrigin = make_double3(lo[0], lo[1], lo[2]);
        g.gridNodeSize = make_int3(n[0], n[1], n[2]);
        g.gridNodeSignedDistance.assign(size_t(n[0]) * size_t(n[1]) * size_t(n[2]), 0.0);

        fundem_shape shape{};
        if (describeShape(shape)) {
            const int status = fundem_levelset_grid(-1, nullptr, &shape, lo, h, n, g.gridNodeSignedDistance.data());
            if (status != FUNDEM_OK) {
                std::cerr << "[LevelSetObject] buildGrid: " << fundem_status_string(status) << std::endl;
                return;
            }
        } else {
            for (int k = 0; k < n[2]; ++k)
                for (int j = 0; j < n[1]; ++j)
                    for (int i = 0; i < n[0]; ++i) {
                        const double3 p = make_double3(lo[0] + double(i) * h, lo[1] + double(j) * h, lo[2] + double(k) * h);
                        double f = 0.0;
                        double3 grad = make_double3(0.0, 0.0, 0.0);
                        evaluateImplicitFunctionValueAndGradient(f, grad, p);
                        const double gn = length(grad);
                        g.gridNodeSignedDistance[linearIndex3D(make_int3(i, j, k), g.gridNodeSize)] =
                            gn > 1e-12 ? f / gn : (f <= 0.0 ? -1.0 : 1.0) * 0.5 * h;
                    }
        }
        gridInfo_ = std::move(g);
    }

    // spacing = largest bounding-box extent / nodes per diameter (:226-254)
    void buildGridByResolution(const int backgroundGridNodesPerParticleDiameter = 50,
                               const int backgroundGridPaddingLayers = 2)
    {
        if (!isValid() || backgroundGridNodesPerParticleDiameter <= 0) return;
        const double3 e = boundingBoxMax() - boundingBoxMin();
        const double d = std::max(e.x, std::max(e.y, e.z));
        if (d <= 0.0) return;
        buildGrid(d / double(backgroundGridNodesPerParticleDiameter), backgroundGridPaddingLayers);
    }

    // <prefix>LSGrid.vtu: one vertex cell per grid node with the signed
    // distance and the node's (i, j, k) (:256-366)
    void outputGridVTU(const std::string& fileNamePrefix) const
    {
        if (!isGridBuilt()) return;
        const int nx = gridInfo_.gridNodeSize.x, ny = gridInfo_.gridNodeSize.y, nz = gridInfo_.gridNodeSize.z;
        const size_t N = size_t(nx) * size_t(ny) * size_t(nz);
        if (nx <= 0 || ny <= 0 || nz <= 0 || gridInfo_.gridNodeSignedDistance.size() != N) return;
        const std::string name = fileNamePrefix + "LSGrid.vtu";
        std::ofstream out(name);
        if (!out) throw std::runtime_error("Cannot open " + name);
        const double h = gridInfo_.gridNodeSpacing;
        const double3 o = gridInfo_.gridOrigin;
        out << "<?xml version=\"1.0\"?>\n"
            << "<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
            << "  <UnstructuredGrid>\n"
            << "    <Piece NumberOfPoints=\"" << N << "\" NumberOfCells=\"" << N << "\">\n"
            << "      <Points>\n        <DataArray type=\"Float32\" NumberOfComponents=\"3\" format=\"ascii\">\n";
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i)
                    out << "          " << float(o.x + double(i) * h) << " " << float(o.y + double(j) * h) << " "
                        << float(o.z + double(k) * h) << "\n";
        out << "        </DataArray>\n      </Points>\n      <Cells>\n"
            << "        <DataArray type=\"Int32\" Name=\"connectivity\" format=\"ascii\">\n";
        for (size_t c = 0; c < N; ++c) out << "          " << c << "\n";
        out << "        </DataArray>\n        <DataArray type=\"Int32\" Name=\"offsets\" format=\"ascii\">\n";
        for (size_t c = 0; c < N; ++c) out << "          " << c + 1 << "\n";
        out << "        </DataArray>\n        <DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n";
        for (size_t c = 0; c < N; ++c) out << "          1\n";
        out << "        </DataArray>\n      </Cells>\n      <PointData Scalars=\"signedDistance\">\n"
            << "        <DataArray type=\"Float32\" Name=\"signedDistance\" format=\"ascii\">\n";
        for (size_t c = 0; c < N; ++c) out << "          " << float(gridInfo_.gridNodeSignedDistance[c]) << "\n";
        out << "        </DataArray>\n"
            << "        <DataArray type=\"Int32\" Name=\"gridIJK\" NumberOfComponents=\"3\" format=\"ascii\">\n";
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) out << "          " << i << " " << j << " " << k << "\n";
        out << "        </DataArray>\n      </PointData>\n    </Piece>\n  </UnstructuredGrid>\n</VTKFile>\n";
    }

    const GridInfo& gridInfo() const { return gridInfo_; }
    GridInfo& gridInfo() { return gridInfo_; }
};

// A closed triangle mesh (:382-955).  The implicit function is the distance
// to the nearest triangle, negative where the winding number says inside.
// The reference finds the nearest triangle through a BVH; the distance is the
// same minimum, which the GPU evaluation takes over all triangles.
class TriangleMeshParticle : public Base
{
protected:
    std::vector<double3> vertexPosition_;
    std::vector<int3> triangleVertexIndex_;
    bool levelSetPositiveInside_{false};
    double3 boundingBoxMin_{0.0, 0.0, 0.0};
    double3 boundingBoxMax_{0.0, 0.0, 0.0};

    static double3 vecMin(const double3& a, const double3& b)
    {
        return make_double3(std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z));
    }
    static double3 vecMax(const double3& a, const double3& b)
    {
        return make_double3(std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z));
    }

    // nearest point of triangle abc to p by Voronoi regions (Ericson,
    // "Real-Time Collision Detection", 2005, section 5.1.5)
    static double3 closestPointOnTriangle(const double3& p, const double3& a, const double3& b, const double3& c)
    {
        const double3 ab = b - a, ac = c - a, ap = p - a;
        const double d1 = dot(ab, ap), d2 = dot(ac, ap);
        if (d1 <= 0.0 && d2 <= 0.0) return a;
        const double3 bp = p - b;
        const double d3 = dot(ab, bp), d4 = dot(ac, bp);
        if (d3 >= 0.0 && d4 <= d3) return b;
        const double vc = d1 * d4 - d3 * d2;
        if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) return a + (d1 / (d1 - d3)) * ab;
        const double3 cp = p - c;
        const double d5 = dot(ab, cp), d6 = dot(ac, cp);
        if (d6 >= 0.0 && d5 <= d6) return c;
        const double vb = d5 * d2 - d1 * d6;
        if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) return a + (d2 / (d2 - d6)) * ac;
        const double va = d3 * d6 - d5 * d4;
        if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0)
            return b + ((d4 - d3) / ((d4 - d3) + (d5 - d6))) * (c - b);
        const double inv = 1.0 / (va + vb + vc);
        return a + ab * (vb * inv) + ac * (vc * inv);
    }

    // signed solid angle of abc seen from p (Van Oosterom and Strackee, 1983)
    static double solidAngleFromPointToTriangle(const double3& p, const double3& a, const double3& b, const double3& c)
    {
        const double3 r0 = a - p, r1 = b - p, r2 = c - p;
        const double l0 = length(r0), l1 = length(r1), l2 = length(r2);
        if (l0 < 1e-30 || l1 < 1e-30 || l2 < 1e-30) return 0.0;
        const double num = dot(r0, cross(r1, r2));
        const double den = l0 * l1 * l2 + dot(r0, r1) * l2 + dot(r1, r2) * l0 + dot(r2, r0) * l1;
        return 2.0 * std::atan2(num, den);
    }

    bool isPointInsideClosedTriangleMesh(const double3& point) const
    {
        if (!isValid()) return false;
        double sum = 0.0;
        for (const int3& t : triangleVertexIndex_)
            sum += solidAngleFromPointToTriangle(point, vertexPosition_[t.x], vertexPosition_[t.y], vertexPosition_[t.z]);
        return std::fabs(sum / (4.0 * pi())) > 0.5;
    }

    void updateBoundingBoxFromMesh()
    {
        if (vertexPosition_.empty()) {
            boundingBoxMin_ = boundingBoxMax_ = make_double3(0.0, 0.0, 0.0);
            return;
        }
        boundingBoxMin_ = boundingBoxMax_ = vertexPosition_[0];
        for (const double3& v : vertexPosition_) {
            boundingBoxMin_ = vecMin(boundingBoxMin_, v);
            boundingBoxMax_ = vecMax(boundingBoxMax_, v);
        }
    }

    void setMeshInternal(const std::vector<double3>& v, const std::vector<int3>& f)
    {
        vertexPosition_ = v;
        triangleVertexIndex_ = f;
        updateBoundingBoxFromMesh();
        clearGrid();
    }

    bool describeMesh(fundem_shape& s) const
    {
        s.kind = FUNDEM_SHAPE_MESH;
        s.positive_inside = levelSetPositiveInside_ ? 1 : 0;
        s.n_vertices = (int)vertexPosition_.size();
        s.vertices = &vertexPosition_[0].x;
        s.n_triangles = (int)triangleVertexIndex_.size();
        s.triangles = &triangleVertexIndex_[0].x;
        return true;
    }

    bool describeShape(fundem_shape& s) const override
    {
        return typeid(*this) == typeid(TriangleMeshParticle) && describeMesh(s);
    }

public:
    TriangleMeshParticle() = default;
    TriangleMeshParticle(const std::vector<double3>& v, const std::vector<int3>& f)
        : vertexPosition_(v), triangleVertexIndex_(f)
    {
        updateBoundingBoxFromMesh();
    }
    ~TriangleMeshParticle() override = default;

    void setMesh(const std::vector<double3>& v, const std::vector<int3>& f) { setMeshInternal(v, f); }
    void setLevelSetPositiveInside(bool v) { levelSetPositiveInside_ = v; }
    void clearMesh()
    {
        vertexPosition_.clear();
        triangleVertexIndex_.clear();
        updateBoundingBoxFromMesh();
        clearGrid();
    }

    // non-empty, every index in range, no triangle repeating a vertex (:872-886)
    bool isValid() const override
    {
        if (vertexPosition_.empty() || triangleVertexIndex_.empty()) return false;
        const int n = (int)vertexPosition_.size();
        for (const int3& t : triangleVertexIndex_) {
            if (t.x < 0 || t.y < 0 || t.z < 0 || t.x >= n || t.y >= n || t.z >= n) return false;
            if (t.x == t.y || t.y == t.z || t.z == t.x) return false;
        }
        return true;
    }

    void evaluateImplicitFunctionValueAndGradient(double& value, double3& grad, const double3& p) const override
    {
        if (!isValid()) {
            value = 1.0;
            grad = make_double3(0.0, 0.0, 0.0);
            return;
        }
        double best = std::numeric_limits<double>::max();
        double3 cp = p;
        for (const int3& t : triangleVertexIndex_) {
            const double3 q = closestPointOnTriangle(p, vertexPosition_[t.x], vertexPosition_[t.y], vertexPosition_[t.z]);
            const double d2 = lengthSquared(p - q);
            if (d2 < best) {
                best = d2;
                cp = q;
            }
        }
        const double d = length(p - cp);
        const bool inside = isPointInsideClosedTriangleMesh(p);
        value = inside ? -d : d;
        if (d > 1e-30) {
            const double3 u = (p - cp) / d;
            grad = inside ? -u : u;
        } else {
            grad = make_double3(0.0, 0.0, 0.0);
        }
        Utility::applyLevelSetSign(value, grad, levelSetPositiveInside_);
    }

    double3 boundingBoxMin() const override { return boundingBoxMin_; }
    double3 boundingBoxMax() const override { return boundingBoxMax_; }

    const std::vector<double3>& vertexPosition() const { return vertexPosition_; }
    std::vector<double3>& vertexPosition() { return vertexPosition_; }
    const std::vector<int3>& triangleVertexIndex() const { return triangleVertexIndex_; }
    std::vector<int3>& triangleVertexIndex() { return triangleVertexIndex_; }
    const double3& meshBoundingBoxMin() const { return boundingBoxMin_; }
    const double3& meshBoundingBoxMax() const { return boundingBoxMax_; }
};

namespace Detail
{
// the regular icosahedron on the golden-ratio rectangles: 12 corners, 20 faces
inline void icosahedron(std::vector<double3>& v, std::vector<int3>& f)
{
    const double t = 0.5 * (1.0 + std::sqrt(5.0));
    v = {make_double3(-1.0, t, 0.0), make_double3(1.0, t, 0.0),  make_double3(-1.0, -t, 0.0),
         make_double3(1.0, -t, 0.0), make_double3(0.0, -1.0, t), make_double3(0.0, 1.0, t),
         make_double3(0.0, -1.0, -t), make_double3(0.0, 1.0, -t), make_double3(t, 0.0, -1.0),
         make_double3(t, 0.0, 1.0),  make_double3(-t, 0.0, -1.0), make_double3(-t, 0.0, 1.0)};
    static const int faces[20][3] = {{0, 11, 5}, {0, 5, 1},  {0, 1, 7},   {0, 7, 10}, {0, 10, 11},
                                     {1, 5, 9},  {5, 11, 4}, {11, 10, 2}, {10, 7, 6}, {7, 1, 8},
                                     {3, 9, 4},  {3, 4, 2},  {3, 2, 6},   {3, 6, 8},  {3, 8, 9},
                                     {4, 9, 5},  {2, 4, 11}, {6, 2, 10},  {8, 6, 7},  {9, 8, 1}};
    f.clear();
    for (const auto& t3 : faces) f.push_back(make_int3(t3[0], t3[1], t3[2]));
}

// One 1-to-4 split of every triangle.  The midpoint of an edge becomes a new
// vertex the first time a triangle (in order, edges 01, 12, 20) uses it;
// `place` maps the two end points to its position.
template <class Place>
inline void subdivide(std::vector<double3>& v, std::vector<int3>& f, Place place)
{
    std::unordered_map<uint64_t, int> mid;
    mid.reserve(f.size() * 3);
    auto midpoint = [&](int a, int b) {
        const uint64_t key = (uint64_t(uint32_t(std::min(a, b))) << 32) | uint32_t(std::max(a, b));
        const auto it = mid.find(key);
        if (it != mid.end()) return it->second;
        const int id = (int)v.size();
        v.push_back(place(v[std::min(a, b)], v[std::max(a, b)]));
        mid.emplace(key, id);
        return id;
    };
    std::vector<int3> out;
    out.reserve(f.size() * 4);
    for (const int3 t : f) {
        const int m01 = midpoint(t.x, t.y), m12 = midpoint(t.y, t.z), m20 = midpoint(t.z, t.x);
        out.push_back(make_int3(t.x, m01, m20));
        out.push_back(make_int3(t.y, m12, m01));
        out.push_back(make_int3(t.z, m20, m12));
        out.push_back(make_int3(m01, m12, m20));
    }
    f.swap(out);
}

// swap two corners of each triangle whose normal points towards the origin
inline void orientOutward(const std::vector<double3>& v, std::vector<int3>& f)
{
    for (int3& t : f) {
        const double3 centre = (v[t.x] + v[t.y] + v[t.z]) / 3.0;
        const double3 normal = cross(v[t.y] - v[t.x], v[t.z] - v[t.x]);
        if (dot(normal, centre) < 0.0) std::swap(t.y, t.z);
    }
}
}  // namespace Detail

// Superellipsoid (|x/rx|^(2/ee) + |y/ry|^(2/ee))^(ee/en) + |z/rz|^(2/en) = 1
// (:956-1362); the surface mesh is an icosphere of the given subdivision
// level (0..8) pushed radially onto the surface.
class Superellipsoid : public TriangleMeshParticle
{
protected:
    double rx_{1.0}, ry_{1.0}, rz_{1.0}, ee_{1.0}, en_{1.0};
    int subdivisionLevel_{4};

    static int clampSubdivisionLevel(const int level) { return std::max(0, std::min(level, 8)); }
    bool parametersAreValid() const
    {
        return rx_ > 0.0 && ry_ > 0.0 && rz_ > 0.0 && ee_ > 0.0 && en_ > 0.0 && subdivisionLevel_ >= 0;
    }

    // the point of the surface along a direction from the centre
    double3 projectUnitDirectionToSuperellipsoid(const double3& direction) const
    {
        const double l2 = lengthSquared(direction);
        if (l2 <= 1e-30) return make_double3(0.0, 0.0, 0.0);
        const double3 u = direction / std::sqrt(l2);
        const double exy = 2.0 / ee_, ez = 2.0 / en_, eo = ee_ / en_;
        const double tx = Utility::safeAbsPow(std::fabs(u.x / rx_), exy);
        const double ty = Utility::safeAbsPow(std::fabs(u.y / ry_), exy);
        const double tz = Utility::safeAbsPow(std::fabs(u.z / rz_), ez);
        const double m = Utility::safeAbsPow(tx + ty, eo) + tz;
        if (m <= 1e-30) return make_double3(0.0, 0.0, 0.0);
        return u * std::pow(m, -0.5 * en_);
    }

    void rebuildMesh()
    {
        clearMesh();
        if (!parametersAreValid()) return;
        std::vector<double3> v;
        std::vector<int3> f;
        Detail::icosahedron(v, f);
        for (double3& p : v) p = normalize(p);
        Detail::orientOutward(v, f);
        for (int level = 0; level < subdivisionLevel_; ++level) {
            Detail::subdivide(v, f, [](const double3& a, const double3& b) { return normalize(0.5 * (a + b)); });
            Detail::orientOutward(v, f);
        }
        for (double3& p : v) p = projectUnitDirectionToSuperellipsoid(p);
        Detail::orientOutward(v, f);
        setMeshInternal(v, f);
    }

    bool describeShape(fundem_shape& s) const override
    {
        if (typeid(*this) != typeid(Superellipsoid)) return false;
        s.kind = FUNDEM_SHAPE_SUPERELLIPSOID;
        s.positive_inside = levelSetPositiveInside_ ? 1 : 0;
        s.param[0] = rx_;
        s.param[1] = ry_;
        s.param[2] = rz_;
        s.param[3] = ee_;
        s.param[4] = en_;
        return true;
    }

public:
    Superellipsoid() = default;
    Superellipsoid(const double rx, const double ry, const double rz, const double ee, const double en,
                   const int subdivisionLevel = 4)
        : rx_(rx), ry_(ry), rz_(rz), ee_(ee), en_(en), subdivisionLevel_(clampSubdivisionLevel(subdivisionLevel))
    {
        rebuildMesh();
    }
    ~Superellipsoid() override = default;
    Superellipsoid(const Superellipsoid&) = default;
    Superellipsoid(Superellipsoid&&) noexcept = default;
    Superellipsoid& operator=(const Superellipsoid&) = default;
    Superellipsoid& operator=(Superellipsoid&&) noexcept = default;

    void setParams(const double rx, const double ry, const double rz, const double ee, const double en,
                   const int subdivisionLevel = 4)
    {
        rx_ = rx;
        ry_ = ry;
        rz_ = rz;
        ee_ = ee;
        en_ = en;
        subdivisionLevel_ = clampSubdivisionLevel(subdivisionLevel);
        rebuildMesh();
    }
    void setSubdivisionLevel(const int subdivisionLevel)
    {
        subdivisionLevel_ = clampSubdivisionLevel(subdivisionLevel);
        rebuildMesh();
    }

    bool isValid() const override { return parametersAreValid() && TriangleMeshParticle::isValid(); }

    void evaluateImplicitFunctionValueAndGradient(double& value, double3& grad, const double3& p) const override
    {
        if (!parametersAreValid()) {
            value = 1.0;
            grad = make_double3(0.0, 0.0, 0.0);
            return;
        }
        const double ix = 1.0 / rx_, iy = 1.0 / ry_, iz = 1.0 / rz_;
        const double ax = std::fabs(p.x * ix), ay = std::fabs(p.y * iy), az = std::fabs(p.z * iz);
        const double exy = 2.0 / ee_, ez = 2.0 / en_, eo = ee_ / en_;
        const double sxy = Utility::safeAbsPow(ax, exy) + Utility::safeAbsPow(ay, exy);
        value = Utility::safeAbsPow(sxy, eo) + Utility::safeAbsPow(az, ez) - 1.0;
        const double tiny = 1e-30;
        const double outer = Utility::safeAbsPow(std::max(sxy, tiny), eo - 1.0);
        const double dsx = exy * Utility::safeAbsPow(std::max(ax, tiny), exy - 1.0) * Utility::signNoZero(p.x) * ix;
        const double dsy = exy * Utility::safeAbsPow(std::max(ay, tiny), exy - 1.0) * Utility::signNoZero(p.y) * iy;
        const double dz = ez * Utility::safeAbsPow(std::max(az, tiny), ez - 1.0) * Utility::signNoZero(p.z) * iz;
        grad = make_double3(eo * outer * dsx, eo * outer * dsy, dz);
        Utility::applyLevelSetSign(value, grad, levelSetPositiveInside_);
    }

    double3 boundingBoxMin() const override { return make_double3(-rx_, -ry_, -rz_); }
    double3 boundingBoxMax() const override { return make_double3(rx_, ry_, rz_); }

    double rx() const { return rx_; }
    double ry() const { return ry_; }
    double rz() const { return rz_; }
    double ee() const { return ee_; }
    double en() const { return en_; }
};

// Sphere of a radius with an icosphere surface of at least the requested
// number of points, 10 * 4^L + 2 for subdivision level L (:1363-1670)
class Sphere : public TriangleMeshParticle
{
protected:
    double radius_{0.0};
    size_t targetSurfacePointCount_{0};

    static double3 projectPointToSphere(const double3& p, const double r)
    {
        const double l = length(p);
        if (l < 1e-30) return make_double3(0.0, 0.0, 0.0);
        return (r / l) * p;
    }
    static int estimateSubdivisionLevelAtLeast(const size_t target)
    {
        if (target <= 12) return 0;
        for (int level = 0; level <= 12; ++level)
            if (static_cast<size_t>(10.0 * std::pow(4.0, level) + 2.0) >= target) return level;
        return 12;
    }

    void rebuildMesh()
    {
        if (radius_ <= 0.0 || targetSurfacePointCount_ < 4) {
            clearMesh();
            return;
        }
        std::vector<double3> v;
        std::vector<int3> f;
        Detail::icosahedron(v, f);
        const double r = radius_;
        for (double3& p : v) p = projectPointToSphere(p, r);
        const int levels = estimateSubdivisionLevelAtLeast(targetSurfacePointCount_);
        for (int level = 0; level < levels; ++level)
            Detail::subdivide(v, f, [r](const double3& a, const double3& b) { return projectPointToSphere(0.5 * (a + b), r); });
        setMeshInternal(v, f);
    }

    bool describeShape(fundem_shape& s) const override
    {
        if (typeid(*this) != typeid(Sphere)) return false;
        s.kind = FUNDEM_SHAPE_SPHERE;
        s.positive_inside = levelSetPositiveInside_ ? 1 : 0;
        s.param[0] = radius_;
        return true;
    }

public:
    Sphere() = default;
    Sphere(const double radius, const size_t targetSurfacePointCount)
        : radius_(radius), targetSurfacePointCount_(targetSurfacePointCount)
    {
        rebuildMesh();
    }
    ~Sphere() override = default;
    Sphere(const Sphere&) = default;
    Sphere(Sphere&&) noexcept = default;
    Sphere& operator=(const Sphere&) = default;
    Sphere& operator=(Sphere&&) noexcept = default;

    void setParams(const double radius, const size_t targetSurfacePointCount)
    {
        radius_ = radius;
        targetSurfacePointCount_ = targetSurfacePointCount;
        rebuildMesh();
    }
    void clearSphere()
    {
        radius_ = 0.0;
        targetSurfacePointCount_ = 0;
        levelSetPositiveInside_ = false;
        clearMesh();
    }

    bool isValid() const override
    {
        return radius_ > 0.0 && targetSurfacePointCount_ >= 4 && TriangleMeshParticle::isValid();
    }

    void evaluateImplicitFunctionValueAndGradient(double& value, double3& grad, const double3& p) const override
    {
        if (radius_ <= 0.0) {
            value = 1.0;
            grad = make_double3(0.0, 0.0, 0.0);
            return;
        }
        const double d = length(p);
        value = d - radius_;
        if (d > 1e-30) grad = p / d;  // at the centre the caller's gradient is left as it was
        Utility::applyLevelSetSign(value, grad, levelSetPositiveInside_);
    }

    double3 boundingBoxMin() const override { return make_double3(-radius_, -radius_, -radius_); }
    double3 boundingBoxMax() const override { return make_double3(radius_, radius_, radius_); }
    double radius() const { return radius_; }
};

// Box wall of edge lengths lx, ly, lz centred on the origin, positive inside
// (:1672-1875).  The default object has no surface mesh until setParams.
class BoxWall : public TriangleMeshParticle
{
protected:
    double lx_{1.0}, ly_{1.0}, lz_{1.0};

    void rebuildMesh()
    {
        std::vector<double3> v;
        std::vector<int3> f;
        if (lx_ > 0.0 && ly_ > 0.0 && lz_ > 0.0) {
            const double hx = 0.5 * lx_, hy = 0.5 * ly_, hz = 0.5 * lz_;
            // corners: bottom face counter-clockwise from (-,-,-), then the top face
            for (int k = 0; k < 2; ++k) {
                const double z = k ? hz : -hz;
                v.push_back(make_double3(-hx, -hy, z));
                v.push_back(make_double3(hx, -hy, z));
                v.push_back(make_double3(hx, hy, z));
                v.push_back(make_double3(-hx, hy, z));
            }
            // two triangles per face, normals pointing out of the box:
            // -z, +z, -x, +x, -y, +y
            static const int faces[12][3] = {{0, 2, 1}, {0, 3, 2}, {4, 5, 6}, {4, 6, 7}, {0, 7, 3}, {0, 4, 7},
                                             {1, 2, 6}, {1, 6, 5}, {0, 1, 5}, {0, 5, 4}, {3, 7, 6}, {3, 6, 2}};
            for (const auto& t3 : faces) f.push_back(make_int3(t3[0], t3[1], t3[2]));
        }
        setMeshInternal(v, f);
    }

    bool describeShape(fundem_shape& s) const override
    {
        if (typeid(*this) != typeid(BoxWall)) return false;
        s.kind = FUNDEM_SHAPE_BOX;
        s.positive_inside = levelSetPositiveInside_ ? 1 : 0;
        s.param[0] = lx_;
        s.param[1] = ly_;
        s.param[2] = lz_;
        return true;
    }

public:
    BoxWall() { levelSetPositiveInside_ = true; }
    BoxWall(const double lx, const double ly, const double lz) : lx_(lx), ly_(ly), lz_(lz)
    {
        levelSetPositiveInside_ = true;
        rebuildMesh();
    }
    ~BoxWall() override = default;
    BoxWall(const BoxWall&) = default;
    BoxWall(BoxWall&&) noexcept = default;
    BoxWall& operator=(const BoxWall&) = default;
    BoxWall& operator=(BoxWall&&) noexcept = default;

    void setParams(const double lx, const double ly, const double lz)
    {
        lx_ = lx;
        ly_ = ly;
        lz_ = lz;
        rebuildMesh();
        clearGrid();
    }

    bool isValid() const override { return lx_ > 0.0 && ly_ > 0.0 && lz_ > 0.0; }

    void evaluateImplicitFunctionValueAndGradient(double& value, double3& grad, const double3& p) const override
    {
        if (!isValid()) {
            value = 1.0;
            grad = make_double3(0.0, 0.0, 0.0);
            return;
        }
        const double3 hb = make_double3(0.5 * lx_, 0.5 * ly_, 0.5 * lz_);
        const double3 q = make_double3(std::fabs(p.x) - hb.x, std::fabs(p.y) - hb.y, std::fabs(p.z) - hb.z);
        const double3 qo = make_double3(std::max(q.x, 0.0), std::max(q.y, 0.0), std::max(q.z, 0.0));
        const double out = length(qo);
        value = out + std::min(std::max(q.x, std::max(q.y, q.z)), 0.0);
        if (out > 1e-30) {
            grad = qo / out;
            if (p.x < 0.0 && q.x > 0.0) grad.x = -grad.x;
            if (p.y < 0.0 && q.y > 0.0) grad.y = -grad.y;
            if (p.z < 0.0 && q.z > 0.0) grad.z = -grad.z;
        } else {
            const double fx = hb.x - std::fabs(p.x), fy = hb.y - std::fabs(p.y), fz = hb.z - std::fabs(p.z);
            if (fx <= fy && fx <= fz) grad = make_double3(p.x >= 0.0 ? 1.0 : -1.0, 0.0, 0.0);
            else if (fy <= fx && fy <= fz) grad = make_double3(0.0, p.y >= 0.0 ? 1.0 : -1.0, 0.0);
            else grad = make_double3(0.0, 0.0, p.z >= 0.0 ? 1.0 : -1.0);
        }
        Utility::applyLevelSetSign(value, grad, levelSetPositiveInside_);
    }

    double3 boundingBoxMin() const override { return make_double3(-0.5 * lx_, -0.5 * ly_, -0.5 * lz_); }
    double3 boundingBoxMax() const override { return make_double3(0.5 * lx_, 0.5 * ly_, 0.5 * lz_); }
    double lx() const { return lx_; }
    double ly() const { return ly_; }
    double lz() const { return lz_; }
};

// Capped cylinder wall from point A to point B, positive inside (:1877-2137).
// The mesh is (axial segments + 1) rings of circumferential vertices, then the
// two cap centres.  In the end-cap regions the reference's gradient is the
// unnormalised axis vector, so the grid there holds distance / |B - A|.
class CylinderWall : public TriangleMeshParticle
{
protected:
    double3 pointA_{0.0, 0.0, -0.5};
    double3 pointB_{0.0, 0.0, 0.5};
    double radius_{1.0};
    int numSegmentsCircumference_{256};
    int numSegmentsAxial_{1};

    void rebuildMesh()
    {
        std::vector<double3> v;
        std::vector<int3> f;
        if (!isValid()) {
            setMeshInternal(v, f);
            return;
        }
        const int nc = numSegmentsCircumference_, na = numSegmentsAxial_;
        const double3 axis = pointB_ - pointA_;
        const double3 dir = axis / length(axis);
        const double3 helper = std::fabs(dir.x) < 0.9 ? make_double3(1.0, 0.0, 0.0) : make_double3(0.0, 1.0, 0.0);
        const double3 u = normalize(cross(dir, helper));
        const double3 w = normalize(cross(dir, u));
        for (int a = 0; a <= na; ++a) {
            const double3 centre = pointA_ + (double(a) / double(na)) * axis;
            for (int s = 0; s < nc; ++s) {
                const double theta = 2.0 * M_PI * double(s) / double(nc);
                v.push_back(centre + radius_ * (std::cos(theta) * u + std::sin(theta) * w));
            }
        }
        auto ring = [nc](int a, int s) { return a * nc + ((s % nc) + nc) % nc; };
        for (int a = 0; a < na; ++a)
            for (int s = 0; s < nc; ++s) {
                f.push_back(make_int3(ring(a, s), ring(a + 1, s), ring(a + 1, s + 1)));
                f.push_back(make_int3(ring(a, s), ring(a + 1, s + 1), ring(a, s + 1)));
            }
        const int capA = (int)v.size();
        v.push_back(pointA_);
        const int capB = (int)v.size();
        v.push_back(pointB_);
        for (int s = 0; s < nc; ++s) f.push_back(make_int3(capA, ring(0, s + 1), ring(0, s)));
        for (int s = 0; s < nc; ++s) f.push_back(make_int3(capB, ring(na, s), ring(na, s + 1)));
        setMeshInternal(v, f);
    }

    bool describeShape(fundem_shape& s) const override
    {
        if (typeid(*this) != typeid(CylinderWall)) return false;
        s.kind = FUNDEM_SHAPE_CYLINDER;
        s.positive_inside = levelSetPositiveInside_ ? 1 : 0;
        const double p[7] = {pointA_.x, pointA_.y, pointA_.z, pointB_.x, pointB_.y, pointB_.z, radius_};
        for (int k = 0; k < 7; ++k) s.param[k] = p[k];
        return true;
    }

public:
    CylinderWall() { levelSetPositiveInside_ = true; }
    CylinderWall(const double3& pointA, const double3& pointB, const double radius,
                 const int numSegmentsCircumference = 256, const int numSegmentsAxial = 1)
        : pointA_(pointA), pointB_(pointB), radius_(radius),
          numSegmentsCircumference_(std::max(3, numSegmentsCircumference)),
          numSegmentsAxial_(std::max(1, numSegmentsAxial))
    {
        levelSetPositiveInside_ = true;
        rebuildMesh();
    }
    ~CylinderWall() override = default;
    CylinderWall(const CylinderWall&) = default;
    CylinderWall(CylinderWall&&) noexcept = default;
    CylinderWall& operator=(const CylinderWall&) = default;
    CylinderWall& operator=(CylinderWall&&) noexcept = default;

    void setParams(const double3& pointA, const double3& pointB, const double radius,
                   const int numSegmentsCircumference = 256, const int numSegmentsAxial = 1)
    {
        pointA_ = pointA;
        pointB_ = pointB;
        radius_ = radius;
        numSegmentsCircumference_ = std::max(3, numSegmentsCircumference);
        numSegmentsAxial_ = std::max(1, numSegmentsAxial);
        rebuildMesh();
        clearGrid();
    }
    void setMeshResolution(const int numSegmentsCircumference, const int numSegmentsAxial)
    {
        numSegmentsCircumference_ = std::max(3, numSegmentsCircumference);
        numSegmentsAxial_ = std::max(1, numSegmentsAxial);
        rebuildMesh();
        clearGrid();
    }

    bool isValid() const override { return radius_ > 0.0 && length(pointB_ - pointA_) > 1e-30; }

    void evaluateImplicitFunctionValueAndGradient(double& value, double3& grad, const double3& p) const override
    {
        if (!isValid()) {
            value = 1.0;
            grad = make_double3(0.0, 0.0, 0.0);
            return;
        }
        const double3 axis = pointB_ - pointA_;
        const double L = length(axis);
        const double3 dir = axis / L;
        const double3 rel = p - pointA_;
        const double s = dot(rel, dir);
        const double3 onAxis = pointA_ + Utility::clampValue(s, 0.0, L) * dir;
        const bool inRadius = length(cross(rel, dir)) <= radius_;
        const bool inLength = s >= 0.0 && s <= L;
        const bool nearA = s < 0.5 * L;
        if (inRadius && inLength) {
            const double3 radial = p - onAxis;
            const double rs = length(radial) - radius_;
            const double as = nearA ? -s : s - L;
            if (std::fabs(rs) <= std::fabs(as)) {
                value = rs;
                grad = normalize(radial);
            } else {
                value = as;
                grad = nearA ? -axis : axis;
            }
        } else if (!inRadius && inLength) {
            const double3 radial = p - onAxis;
            value = length(radial) - radius_;
            grad = normalize(radial);
        } else if (!inRadius && !inLength) {
            const double3 rim = onAxis + normalize(rel - s * dir) * radius_;
            value = length(p - rim);
            grad = normalize(p - rim);
        } else {
            value = s < 0.0 ? -s : s - L;
            grad = s < 0.0 ? -axis : axis;
        }
        Utility::applyLevelSetSign(value, grad, levelSetPositiveInside_);
    }

    double3 boundingBoxMin() const override
    {
        return make_double3(std::min(pointA_.x, pointB_.x) - radius_, std::min(pointA_.y, pointB_.y) - radius_,
                            std::min(pointA_.z, pointB_.z) - radius_);
    }
    double3 boundingBoxMax() const override
    {
        return make_double3(std::max(pointA_.x, pointB_.x) + radius_, std::max(pointA_.y, pointB_.y) + radius_,
                            std::max(pointA_.z, pointB_.z) + radius_);
    }

    const double3& pointA() const { return pointA_; }
    const double3& pointB() const { return pointB_; }
    double radius() const { return radius_; }
};

}  // namespace LevelSetObject
