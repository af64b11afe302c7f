// SpherePack -- sphere centres and radii in a box, with the class name,
// members, method names, arguments and results of the reference's
// kernel/Packing.h: random sequential addition with the largest spheres
// first (:24-118), a simple cubic lattice (:123-142) and a hexagonal close
// packing (:147-182).  Host code only.
//
// A seed gives the reference's packing: the same std::mt19937 stream is
// consumed in the same order (every radius first, then three uniforms per
// placement attempt, the z uniform first: the reference draws them inside
// one make_double3 call, whose arguments GCC evaluates last to first), and
// candidate centres and the lattice coordinates are formed with the same
// floating-point operations.  Placed spheres are binned in cells of twice the
// largest radius, so a candidate is compared with the spheres of the 27
// cells around it, which holds every sphere it can overlap.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <functional>
#include <random>
#include <unordered_map>
#include <vector>

#include "CUDAKernelFunction/myUtility/myVec.h"

class SpherePack
{
public:
    std::vector<double3> centers;
    std::vector<double> radii;

public:
    void buildNonOverlappingInBox_LargeFirst(const double3 boxMin, const double3 boxMax, const int nSpheres,
                                             const double rMin, const double rMax, const uint32_t seed = 12345u,
                                             const int maxAttemptsPerSphere = 2000)
    {
        centers.clear();
        radii.clear();
        if (nSpheres <= 0 || rMin <= 0.0 || rMax < rMin) return;
        const double3 lo = make_double3(std::min(boxMin.x, boxMax.x), std::min(boxMin.y, boxMax.y),
                                        std::min(boxMin.z, boxMax.z));
        const double3 hi = make_double3(std::max(boxMin.x, boxMax.x), std::max(boxMin.y, boxMax.y),
                                        std::max(boxMin.z, boxMax.z));
        std::mt19937 rng(seed);
        std::uniform_real_distribution<double> unit(0.0, 1.0);
        std::uniform_real_distribution<double> radius(rMin, rMax);
        std::vector<double> order((size_t)nSpheres);
        for (double& r : order) r = radius(rng);
        std::sort(order.begin(), order.end(), std::greater<double>());

        const double cell = 2.0 * rMax;
        std::unordered_map<uint64_t, std::vector<int>> bins;
        bins.reserve((size_t)nSpheres * 2);
        auto cellOf = [&](const double3& p, int c[3]) {
            c[0] = (int)std::floor((p.x - lo.x) / cell);
            c[1] = (int)std::floor((p.y - lo.y) / cell);
            c[2] = (int)std::floor((p.z - lo.z) / cell);
        };
        // 21 bits per axis, offset so that cells just outside the box stay
        // distinct
        auto key = [](int x, int y, int z) {
            const uint64_t m = (1ull << 21) - 1;
            return ((uint64_t)(x + (1 << 20)) & m) << 42 | ((uint64_t)(y + (1 << 20)) & m) << 21 |
                   ((uint64_t)(z + (1 << 20)) & m);
        };
        auto clear = [&](const double3& p, double r) {
            int c[3];
            cellOf(p, c);
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        const auto it = bins.find(key(c[0] + dx, c[1] + dy, c[2] + dz));
                        if (it == bins.end()) continue;
                        for (const int id : it->second) {
                            const double3 d = p - centers[(size_t)id];
                            const double rr = r + radii[(size_t)id];
                            if (dot(d, d) < rr * rr) return false;
                        }
                    }
            return true;
        };
        for (const double r : order) {
            for (int attempt = 0; attempt < maxAttemptsPerSphere; ++attempt) {
                const double uz = unit(rng);
                const double uy = unit(rng);
                const double ux = unit(rng);
                const double3 p = make_double3((lo.x + r) + ux * (hi.x - lo.x - 2 * r),
                                               (lo.y + r) + uy * (hi.y - lo.y - 2 * r),
                                               (lo.z + r) + uz * (hi.z - lo.z - 2 * r));
                if (!clear(p, r)) continue;
                int c[3];
                cellOf(p, c);
                bins[key(c[0], c[1], c[2])].push_back((int)centers.size());
                centers.push_back(p);
                radii.push_back(r);
                break;
            }
        }
    }

    // Simple cubic lattice of spacing 2r from boxMin + r, while a sphere fits
    // below boxMax; coordinates advance by repeated addition, as the
    // reference's loops do.
    void buildRegularInBox(const double3 boxMin, const double3 boxMax, const double r)
    {
        centers.clear();
        radii.clear();
        if (r <= 0.0) return;
        const double step = 2.0 * r;
        for (double z = boxMin.z + r; z <= boxMax.z - r; z += step)
            for (double y = boxMin.y + r; y <= boxMax.y - r; y += step)
                for (double x = boxMin.x + r; x <= boxMax.x - r; x += step) {
                    centers.push_back(make_double3(x, y, z));
                    radii.push_back(r);
                }
    }

    // Hexagonal close packing: rows 2r apart in x, sqrt(3) r in y, layers
    // sqrt(8/3) r in z; odd rows and odd layers start r further along x.
    void buildHexInBox(const double3 boxMin, const double3 boxMax, const double r)
    {
        centers.clear();
        radii.clear();
        if (r <= 0.0) return;
        const double sx = 2 * r, sy = std::sqrt(3.0) * r, sz = std::sqrt(8.0 / 3.0) * r;
        int layer = 0;
        for (double z = boxMin.z + r; z <= boxMax.z - r; z += sz, ++layer) {
            int row = 0;
            for (double y = boxMin.y + r; y <= boxMax.y - r; y += sy, ++row) {
                double x0 = boxMin.x + r;
                if (row % 2 == 1) x0 += r;
                if (layer % 2 == 1) x0 += r;
                for (double x = x0; x <= boxMax.x - r; x += sx) {
                    centers.push_back(make_double3(x, y, z));
                    radii.push_back(r);
                }
            }
        }
    }
};
