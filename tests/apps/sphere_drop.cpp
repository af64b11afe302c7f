// A sphere dropped on a plane wall, written against the LSSolver call
// surface (kernel/LSSolver.h) to check that such an app builds and runs on
// libfundem_b200.  Prints the sphere's final position and velocity.
//
//   sphere_drop <outdir> [hover]
//
// With "hover", an addExternalForceTorque hook (a CUDA kernel in
// sphere_hover.cu) cancels gravity, so the sphere stays where it starts.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "kernel/LSSolver.h"

extern "C" void launchAddConstantForce(double3* force, int index, double3 f, cudaStream_t stream);

struct DropSolver : public LSSolver {
    DropSolver(const std::string& dir, bool hover, double weight) : LSSolver(dir), hover_(hover), weight_(weight) {}
    void addExternalForceTorque(const double) override
    {
        if (hover_) launchAddConstantForce(getLSParticle().force(), 0, make_double3(0., 0., weight_), 0);
    }
    double3 finalPosition() { return getLSParticle().positionHostRef()[0]; }
    double3 finalVelocity() { return getLSParticle().velocityHostRef()[0]; }
    bool hover_;
    double weight_;
};

int main(int argc, char** argv)
{
    const std::string out = argc > 1 ? argv[1] : "sphere_drop";
    const bool hover = argc > 2 && std::strcmp(argv[2], "hover") == 0;
    const double r = 0.01, rho = 2000.0, g = 9.81, h0 = 0.05;
    const double m = 4.0 / 3.0 * pi() * r * r * r * rho;
    const double tc = 0.005;  // contact duration
    const double kn = 0.5 * m * pi() * pi() / (tc * tc);
    DropSolver s(out, hover, m * g);

    // sphere template: signed distance on a 13^3 grid, a ring-and-pole node set
    const double h = r / 5.0;
    const int3 n3 = make_int3(13, 13, 13);
    const double3 o = make_double3(-6 * h, -6 * h, -6 * h);
    std::vector<double> sdf(13 * 13 * 13);
    for (int z = 0; z < 13; ++z)
        for (int y = 0; y < 13; ++y)
            for (int x = 0; x < 13; ++x)
                sdf[linearIndex3D(make_int3(x, y, z), n3)] = length(o + make_double3(x, y, z) * h) - r;
    std::vector<double3> nodes;
    for (int i = 0; i <= 8; ++i)
        for (int j = 0; j < 12; ++j) {
            const double th = pi() * i / 8.0, ph = 2.0 * pi() * j / 12.0;
            nodes.push_back(make_double3(r * std::sin(th) * std::cos(ph), r * std::sin(th) * std::sin(ph),
                                         r * std::cos(th)));
        }
    const double I = 0.4 * m * r * r;
    s.addParticleMaterial(kn, 0.0, 0.0, 1.0);
    s.addParticleGeometry(m, make_symMatrix(I, I, I, 0, 0, 0), o, h, n3, sdf, nodes, std::vector<int3>());
    s.addParticle(make_double3(0, 0, h0), make_double3(0, 0, 0), make_double3(0, 0, 0), make_quaternion(1, 0, 0, 0),
                  0, 0);

    // plane wall z = 0 as a 2 x 2 x 2 linear field
    const double L = 1.0;
    std::vector<double> plane(8);
    const double3 po = make_double3(-0.5 * L, -0.5 * L, -0.5 * L);
    for (int z = 0; z < 2; ++z)
        for (int y = 0; y < 2; ++y)
            for (int x = 0; x < 2; ++x)
                plane[linearIndex3D(make_int3(x, y, z), make_int3(2, 2, 2))] = po.z + z * L;
    std::vector<double3> pnodes = {make_double3(-0.4, -0.4, 0), make_double3(0.4, -0.4, 0),
                                   make_double3(0.4, 0.4, 0), make_double3(-0.4, 0.4, 0)};
    s.addWallMaterial(0.0, 1.0);
    s.addWallGeometry(po, L, make_int3(2, 2, 2), plane, pnodes, std::vector<int3>());
    s.addWall(make_double3(0, 0, 0), make_double3(0, 0, 0), make_double3(0, 0, 0), make_quaternion(1, 0, 0, 0), 0,
              0);

    const double dt = tc / 50.0;
    s.solve(make_double3(-0.5, -0.5, -0.1), make_double3(0.5, 0.5, 0.2), make_double3(0, 0, -g), dt, 0.15, 3, argc,
            argv);
    const double3 x = s.finalPosition(), v = s.finalVelocity();
    std::printf("%.17g %.17g %.17g %.17g %.17g %.17g\n", x.x, x.y, x.z, v.x, v.y, v.z);
    return 0;
}
