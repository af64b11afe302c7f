// SpherePacking:: -- initial particle positions: lattices in a box and random
// non-overlapping packings in a box or a cylinder, with the function names,
// arguments and results of the reference's kernel/helper/SpherePackingGenerator.h.
//
// The random packings draw from std::mt19937 in the reference's order (all
// radii first, then three uniforms per placement attempt) so a seed gives the
// same packing; the overlap test uses a dense cell array instead of a hash map,
// which changes nothing in the result.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <functional>
#include <random>
#include <stdexcept>
#include <vector>

#include "../CUDAKernelFunction/myUtility/myVec.h"

namespace SpherePacking
{

struct Pack {
    std::vector<double3> centers;
    std::vector<double> radii;
};

namespace Utility
{
inline double3 sortedMin(const double3& a, const double3& b)
{
    return make_double3(std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z));
}
inline double3 sortedMax(const double3& a, const double3& b)
{
    return make_double3(std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z));
}
inline bool isSphereInsideBox(const double3& c, const double r, const double3& boxMin, const double3& boxMax)
{
    return c.x - r >= boxMin.x && c.x + r <= boxMax.x && c.y - r >= boxMin.y && c.y + r <= boxMax.y &&
           c.z - r >= boxMin.z && c.z + r <= boxMax.z;
}
}  // namespace Utility

namespace Detail
{
// Placed spheres binned in cells of edge 2 rMax over a box: a new sphere can
// only overlap spheres in its own and the 26 neighbouring cells.
class CellBins
{
public:
    CellBins(const double3& origin, const double3& extent, double cell) : o_(origin), cell_(cell)
    {
        n_[0] = std::max(1, (int)std::floor(extent.x / cell) + 1);
        n_[1] = std::max(1, (int)std::floor(extent.y / cell) + 1);
        n_[2] = std::max(1, (int)std::floor(extent.z / cell) + 1);
        bins_.resize(size_t(n_[0]) * n_[1] * n_[2]);
    }
    void cellOf(const double3& p, int c[3]) const
    {
        c[0] = (int)std::floor((p.x - o_.x) / cell_);
        c[1] = (int)std::floor((p.y - o_.y) / cell_);
        c[2] = (int)std::floor((p.z - o_.z) / cell_);
    }
    void insert(const double3& p, int id)
    {
        int c[3];
        cellOf(p, c);
        for (int a = 0; a < 3; ++a) c[a] = std::min(std::max(c[a], 0), n_[a] - 1);
        bins_[(size_t(c[2]) * n_[1] + c[1]) * n_[0] + c[0]].push_back(id);
    }
    // true when the sphere (p, r) overlaps a placed one: |d| < r + r_placed
    bool overlaps(const double3& p, double r, const Pack& pk) const
    {
        int c[3];
        cellOf(p, c);
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int x = c[0] + dx, y = c[1] + dy, z = c[2] + dz;
                    if (x < 0 || y < 0 || z < 0 || x >= n_[0] || y >= n_[1] || z >= n_[2]) continue;
                    for (int id : bins_[(size_t(z) * n_[1] + y) * n_[0] + x]) {
                        const double3 d = p - pk.centers[(size_t)id];
                        const double rr = r + pk.radii[(size_t)id];
                        if (dot(d, d) < rr * rr) return true;
                    }
                }
        return false;
    }

private:
    double3 o_;
    double cell_;
    int n_[3];
    std::vector<std::vector<int>> bins_;
};

// nSpheres radii uniform in [rMin, rMax), largest first
inline std::vector<double> drawRadiiLargestFirst(std::mt19937& rng, int n, double rMin, double rMax)
{
    std::uniform_real_distribution<double> dist(rMin, rMax);
    std::vector<double> r;
    r.reserve((size_t)n);
    for (int i = 0; i < n; ++i) r.push_back(dist(rng));
    std::sort(r.begin(), r.end(), std::greater<double>());
    return r;
}
}  // namespace Detail

// Random sequential addition in a box (SpherePackingGenerator.h:75-216): radii
// largest first; each sphere tries up to maxAttemptsPerSphere uniform centres
// that keep it inside the box and is dropped when none is free.
inline Pack buildNonOverlappingInBox_LargeFirst(const double3 boxMin, const double3 boxMax, const int nSpheres,
                                                const double rMin, const double rMax, const uint32_t seed = 12345u,
                                                const int maxAttemptsPerSphere = 2000)
{
    Pack out;
    if (nSpheres <= 0 || rMin <= 0.0 || rMax < rMin) return out;
    const double3 lo = Utility::sortedMin(boxMin, boxMax);
    const double3 hi = Utility::sortedMax(boxMin, boxMax);
    const double3 ext = hi - lo;
    if (ext.x < 2.0 * rMin || ext.y < 2.0 * rMin || ext.z < 2.0 * rMin) return out;
    std::mt19937 rng(seed);
    std::uniform_real_distribution<double> u01(0.0, 1.0);
    const std::vector<double> radii = Detail::drawRadiiLargestFirst(rng, nSpheres, rMin, rMax);
    Detail::CellBins bins(lo, ext, 2.0 * rMax);
    out.centers.reserve((size_t)nSpheres);
    out.radii.reserve((size_t)nSpheres);
    for (const double r : radii) {
        if (ext.x < 2.0 * r || ext.y < 2.0 * r || ext.z < 2.0 * r) continue;
        for (int attempt = 0; attempt < maxAttemptsPerSphere; ++attempt) {
            const double x0 = lo.x + r, y0 = lo.y + r, z0 = lo.z + r;
            const double x1 = hi.x - r, y1 = hi.y - r, z1 = hi.z - r;
            // The reference draws the three uniforms inside one make_double3
            // call; GCC evaluates those arguments last to first, so z takes
            // the first draw.  The order is fixed here to give its packings.
            const double uz = u01(rng);
            const double uy = u01(rng);
            const double ux = u01(rng);
            const double3 c = make_double3(x0 + ux * (x1 - x0), y0 + uy * (y1 - y0), z0 + uz * (z1 - z0));
            if (bins.overlaps(c, r, out)) continue;
            bins.insert(c, (int)out.centers.size());
            out.centers.push_back(c);
            out.radii.push_back(r);
            break;
        }
    }
    return out;
}

// Random sequential addition in the cylinder from A to B of the given radius
// (:218-410).  A candidate centre is uniform over the disc of radius R - r
// (r_disc = (R - r) sqrt(u)) and along the axis, then kept only if the sphere
// lies inside the cylinder and overlaps no placed sphere.
inline Pack buildNonOverlappingInCylinder_LargeFirst(const double3 cylinderPointA, const double3 cylinderPointB,
                                                     const double cylinderRadius, const int nSpheres,
                                                     const double rMin, const double rMax,
                                                     const uint32_t seed = 12345u,
                                                     const int maxAttemptsPerSphere = 2000)
{
    Pack out;
    if (nSpheres <= 0 || rMin <= 0.0 || rMax < rMin || cylinderRadius <= 0.0) return out;
    const double3 axis = cylinderPointB - cylinderPointA;
    const double L = length(axis);
    if (L <= 0.0 || L < 2.0 * rMin || cylinderRadius < rMin) return out;
    const double3 dir = axis / L;
    const double3 helper = std::fabs(dir.x) < 0.9 ? make_double3(1.0, 0.0, 0.0) : make_double3(0.0, 1.0, 0.0);
    const double3 eu = normalize(cross(dir, helper));
    const double3 ev = normalize(cross(dir, eu));
    std::mt19937 rng(seed);
    std::uniform_real_distribution<double> u01(0.0, 1.0);
    const std::vector<double> radii = Detail::drawRadiiLargestFirst(rng, nSpheres, rMin, rMax);
    const double R = cylinderRadius;
    const double3 boxLo = make_double3(std::min(cylinderPointA.x, cylinderPointB.x) - R,
                                       std::min(cylinderPointA.y, cylinderPointB.y) - R,
                                       std::min(cylinderPointA.z, cylinderPointB.z) - R);
    const double3 boxHi = make_double3(std::max(cylinderPointA.x, cylinderPointB.x) + R,
                                       std::max(cylinderPointA.y, cylinderPointB.y) + R,
                                       std::max(cylinderPointA.z, cylinderPointB.z) + R);
    Detail::CellBins bins(boxLo, boxHi - boxLo, 2.0 * rMax);
    auto inside = [&](const double3& c, double r) {
        const double3 rel = c - cylinderPointA;
        const double s = dot(rel, dir);
        if (s < r || s > L - r) return false;
        const double3 radial = c - (cylinderPointA + s * dir);
        const double allowed = R - r;
        if (allowed < 0.0) return false;
        return dot(radial, radial) <= allowed * allowed;
    };
    out.centers.reserve((size_t)nSpheres);
    out.radii.reserve((size_t)nSpheres);
    for (const double r : radii) {
        if (L < 2.0 * r || R < r) continue;
        for (int attempt = 0; attempt < maxAttemptsPerSphere; ++attempt) {
            const double uDisc = u01(rng);
            const double uAngle = u01(rng);
            const double rd = (R - r) * std::sqrt(uDisc);
            const double phi = 2.0 * pi() * uAngle;
            const double cu = rd * std::cos(phi), cv = rd * std::sin(phi);
            const double s = r + u01(rng) * ((L - r) - r);
            const double3 c = cylinderPointA + s * dir + cu * eu + cv * ev;
            if (!inside(c, r) || bins.overlaps(c, r, out)) continue;
            bins.insert(c, (int)out.centers.size());
            out.centers.push_back(c);
            out.radii.push_back(r);
            break;
        }
    }
    return out;
}

namespace Detail
{
inline void checkLattice(const double3& boxMin, const double3& boxMax, double r)
{
    if (r <= 0.0) throw std::runtime_error("sphereRadius must be positive.");
    if (boxMax.x <= boxMin.x || boxMax.y <= boxMin.y || boxMax.z <= boxMin.z)
        throw std::runtime_error("Invalid box: boxMax must be larger than boxMin.");
}
}  // namespace Detail

// simple cubic lattice of spacing 2r from boxMin + r, x fastest (:412-460);
// the loop counters accumulate, as in the reference, with a 1e-12 tolerance
// at the far wall
inline Pack buildRegularInBox(const double3 boxMin, const double3 boxMax, const double sphereRadius)
{
    Detail::checkLattice(boxMin, boxMax, sphereRadius);
    Pack pack;
    const double r = sphereRadius, eps = 1.0e-12, step = 2.0 * r;
    const double3 lo = make_double3(boxMin.x + r, boxMin.y + r, boxMin.z + r);
    const double3 hi = make_double3(boxMax.x - r, boxMax.y - r, boxMax.z - r);
    if (lo.x > hi.x || lo.y > hi.y || lo.z > hi.z) return pack;
    for (double z = lo.z; z <= hi.z + eps; z += step)
        for (double y = lo.y; y <= hi.y + eps; y += step)
            for (double x = lo.x; x <= hi.x + eps; x += step) {
                pack.centers.push_back(make_double3(x, y, z));
                pack.radii.push_back(r);
            }
    return pack;
}

// hexagonal close packing (:462-553): rows sqrt(3) r apart, layers
// sqrt(8/3) r apart; odd rows shift by r in x, odd layers by r in x and
// sqrt(3) r / 3 in y; spheres that would cross the box are left out
inline Pack buildHexInBox(const double3 boxMin, const double3 boxMax, const double sphereRadius)
{
    Detail::checkLattice(boxMin, boxMax, sphereRadius);
    Pack pack;
    const double r = sphereRadius, eps = 1.0e-12;
    const double3 lo = make_double3(boxMin.x + r, boxMin.y + r, boxMin.z + r);
    const double3 hi = make_double3(boxMax.x - r, boxMax.y - r, boxMax.z - r);
    if (lo.x > hi.x || lo.y > hi.y || lo.z > hi.z) return pack;
    const double dx = 2.0 * r, dy = std::sqrt(3.0) * r, dz = std::sqrt(8.0 / 3.0) * r;
    const double layerShiftY = std::sqrt(3.0) * r / 3.0;
    int layer = 0;
    for (double z = lo.z; z <= hi.z + eps; z += dz, ++layer) {
        const bool oddLayer = (layer % 2) == 1;
        int row = 0;
        for (double y = lo.y + (oddLayer ? layerShiftY : 0.0); y <= hi.y + eps; y += dy, ++row) {
            double x0 = lo.x;
            if (row % 2 == 1) x0 += r;
            if (oddLayer) x0 += r;
            for (double x = x0; x <= hi.x + eps; x += dx) {
                const double3 c = make_double3(x, y, z);
                if (!Utility::isSphereInsideBox(c, r, boxMin, boxMax)) continue;
                pack.centers.push_back(c);
                pack.radii.push_back(r);
            }
        }
    }
    return pack;
}

}  // namespace SpherePacking
