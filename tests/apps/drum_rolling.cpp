// Superellipsoids settling in a closed cylindrical drum that then turns about
// its axis, written against the LSSolver call surface and its helper
// namespaces: SpherePacking:: places the particles, LevelSetObject:: builds
// one superellipsoid template per particle and the drum's CylinderWall grid.
//
//   drum_rolling <outdir> [n_max]
//
// Writes <outdir>/state_<phase>.txt after the settling phase (0) and after
// the turning phase (1): one line per particle, position, velocity, mass.
#include <cmath>
#include <cstdio>
#include <filesystem>
#include <cstdlib>
#include <fstream>
#include <random>
#include <string>
#include <vector>

#include "kernel/LSSolver.h"
#include "kernel/helper/LevelSetObjectGenerator.h"
#include "kernel/helper/SpherePackingGenerator.h"

struct Drum : public LSSolver {
    explicit Drum(const std::string& dir) : LSSolver(dir) {}
    bool writeState(const std::string& file, const std::vector<double>& mass)
    {
        const std::vector<double3>& x = getLSParticle().positionHostRef();
        const std::vector<double3>& v = getLSParticle().velocityHostRef();
        std::ofstream f(file);
        if (!f) return false;
        f.precision(17);
        for (size_t i = 0; i < x.size(); ++i)
            f << x[i].x << ' ' << x[i].y << ' ' << x[i].z << ' ' << v[i].x << ' ' << v[i].y << ' ' << v[i].z << ' '
              << mass[i] << '\n';
        return bool(f);
    }
};

int main(int argc, char** argv)
{
    const std::string out = argc > 1 ? argv[1] : "drum";
    const int nMax = argc > 2 ? std::atoi(argv[2]) : 40;
    const double L = 0.5, R = 1.0, density = 1000.0;
    const double3 A = make_double3(-L, 0.0, 0.0), B = make_double3(L, 0.0, 0.0);

    std::filesystem::create_directories(out);
    Drum drum(out);
    drum.addParticleMaterial(6.0e5, 1.8e5, 0.5, 0.5);
    drum.addWallMaterial(0.5, 0.5);

    const SpherePacking::Pack pack = SpherePacking::buildNonOverlappingInCylinder_LargeFirst(A, B, R, nMax, 0.15, 0.3);
    // four shape families, scaled to each packing sphere
    const double shapes[4][5] = {
        {0.4, 1.0, 0.8, 0.4, 1.6}, {0.5, 0.7, 1.0, 1.4, 1.2}, {1.0, 1.0, 1.0, 1.0, 0.5}, {0.8, 0.9, 1.0, 1.0, 1.0}};
    std::mt19937 rng(7);
    std::vector<double> mass;
    for (size_t i = 0; i < pack.centers.size(); ++i) {
        const double* s = shapes[i % 4];
        const double k = 0.7 * pack.radii[i];
        LevelSetObject::Superellipsoid se;
        se.setParams(s[0] * k, s[1] * k, s[2] * k, s[3], s[4], 3);
        se.buildGridByResolution(30);
        const LevelSetObject::GridInfo& g = se.gridInfo();
        double m = 0.0, c[3], I[6];
        fundem_mass_properties(density, &g.gridOrigin.x, g.gridNodeSpacing, &g.gridNodeSize.x,
                               g.gridNodeSignedDistance.data(), &m, c, I);
        mass.push_back(m);
        std::uniform_real_distribution<double> u(-1.0, 1.0);
        quaternion q = make_quaternion(1.0, 0.3 * u(rng), 0.3 * u(rng), 0.3 * u(rng));
        const double qn = std::sqrt(q.q0 * q.q0 + q.q1 * q.q1 + q.q2 * q.q2 + q.q3 * q.q3);
        q = make_quaternion(q.q0 / qn, q.q1 / qn, q.q2 / qn, q.q3 / qn);
        drum.addParticleCluster({pack.centers[i]}, {make_double3(0, 0, 0)}, {make_double3(0, 0, 0)}, {q}, 0, density,
                                g.gridOrigin, g.gridNodeSpacing, g.gridNodeSize, g.gridNodeSignedDistance,
                                se.vertexPosition(), se.triangleVertexIndex());
    }

    LevelSetObject::CylinderWall wall;
    wall.setParams(A, B, R, 96, 2);
    wall.buildGridByResolution(60);
    const LevelSetObject::GridInfo& wg = wall.gridInfo();
    drum.addWallGeometry(wg.gridOrigin, wg.gridNodeSpacing, wg.gridNodeSize, wg.gridNodeSignedDistance,
                         wall.vertexPosition(), wall.triangleVertexIndex());
    drum.addWall(make_double3(0, 0, 0), make_double3(0, 0, 0), make_double3(0, 0, 0), make_quaternion(1, 0, 0, 0), 0, 0);

    const double3 lo = make_double3(-L, -2.0 * R, -2.0 * R), hi = make_double3(L, 2.0 * R, 2.0 * R);
    const double3 gravity = make_double3(0.0, 0.0, -9.81);
    drum.solve(lo, hi, gravity, 1.0e-4, 1.0, 2, argc, argv);
    if (!drum.writeState(out + "/state_0.txt", mass)) return 1;
    drum.setFixedAngularVelocityToWall(0, make_double3(pi(), 0.0, 0.0));
    drum.solve(lo, hi, gravity, 1.0e-4, 0.5, 2, argc, argv);
    if (!drum.writeState(out + "/state_1.txt", mass)) return 1;
    std::printf("particles %zu\n", pack.centers.size());
    return 0;
}
