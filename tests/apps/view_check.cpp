// The device getters of SolidInteraction and VBondedInteraction, used from an
// addExternalForceTorque hook as an app written against the reference's
// LSSolver would: a small pile of spheres on a plane wall, two of them bonded,
// and at every hook the device arrays (contactPoint(), masterID(),
// slaveID(), slidingSpring(), contactOverlap(), activated(), B1(), Un(), the
// body-frame vectors, ...) are copied back and compared with the host
// getters.  Prints "views ok <checks>" or the first mismatch.
//
//   view_check <outdir>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "kernel/LSSolver.h"

template <class T>
static std::vector<T> fetch(const T* d, size_t n)
{
    std::vector<T> h(n);
    if (n) cudaMemcpy(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost);
    return h;
}

struct ViewSolver : public LSSolver {
    explicit ViewSolver(const std::string& dir) : LSSolver(dir) {}
    int checks = 0, failures = 0;
    void fail(const char* what, size_t i)
    {
        if (failures++ == 0) std::printf("mismatch %s at %zu\n", what, i);
    }
    void addExternalForceTorque(const double) override
    {
        SolidInteraction& P = getLSParticleInteraction();
        const size_t n = P.numPair_device();
        const std::vector<int> hm = P.masterIDHostRef(), hs = P.slaveIDHostRef();
        const std::vector<double3> hp = P.contactPointHostRef(), hsp = P.slidingSpringHostRef();
        const std::vector<double> ho = P.contactOverlapHostRef();
        const std::vector<int> dm = fetch(P.masterID(), n), ds = fetch(P.slaveID(), n);
        const std::vector<double3> dp = fetch(P.contactPoint(), n), dsp = fetch(P.slidingSpring(), n);
        const std::vector<double> dov = fetch(P.contactOverlap(), n);
        for (size_t i = 0; i < n; ++i) {
            if (dm[i] != hm[i] || ds[i] != hs[i]) fail("ids", i);
            if (dp[i].x != hp[i].x || dp[i].y != hp[i].y || dp[i].z != hp[i].z) fail("point", i);
            if (dsp[i].x != hsp[i].x || dsp[i].y != hsp[i].y || dsp[i].z != hsp[i].z) fail("spring", i);
            if (dov[i] != ho[i]) fail("overlap", i);
        }
        VBondedInteraction& B = getLSParticleBondedInteraction();
        const size_t nb = B.numPair_device();
        const std::vector<int> ha = B.activatedHostRef();
        const std::vector<double> he = B.energyAndStressHostRef();
        const std::vector<int> da = fetch(B.activated(), nb), dmo = fetch(B.masterObjectID(), nb);
        const std::vector<double> dun = fetch(B.Un(), nb), db1 = fetch(B.B1(), nb), dss = fetch(B.maxShearStress(), nb);
        const std::vector<double3> dn1 = fetch(B.masterVBondPointLocalVectorN1(), nb);
        for (size_t i = 0; i < nb; ++i) {
            if (da[i] != ha[i]) fail("activated", i);
            if (dmo[i] != 0) fail("bond master", i);
            if (dun[i] != he[6 * i] || dss[i] != he[6 * i + 5]) fail("bond energies", i);
            if (!(db1[i] > 0.0)) fail("B1", i);
            if (std::fabs(dn1[i].x * dn1[i].x + dn1[i].y * dn1[i].y + dn1[i].z * dn1[i].z - 1.0) > 1e-12)
                fail("frame", i);
        }
        checks += (int)(n + nb);
    }
};

int main(int argc, char** argv)
{
    const std::string out = argc > 1 ? argv[1] : "view_check";
    const double r = 0.01, rho = 2000.0;
    const double m = 4.0 / 3.0 * pi() * r * r * r * rho;
    ViewSolver s(out);
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
    s.addParticleMaterial(2e4, 1.6e4, 0.5, 0.5);
    s.addParticleGeometry(m, make_symMatrix(I, I, I, 0, 0, 0), o, h, n3, sdf, nodes, std::vector<int3>());
    // a 3 x 3 x 2 pile, slightly overlapping, on the floor
    int id = 0;
    for (int k = 0; k < 2; ++k)
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i, ++id)
                s.addParticle(make_double3((i - 1) * 1.96 * r, (j - 1) * 1.96 * r, r * 0.99 + k * 1.96 * r),
                              make_double3(0.01 * (id % 3 - 1), 0.0, 0.0), make_double3(0, 0, 0),
                              make_quaternion(1, 0, 0, 0), 0, 0);
    s.addBondedInteraction(0, 1, make_double3(-0.98 * r, -1.96 * r, 0.99 * r), make_double3(1, 0, 0), 0.3 * r,
                           1.96 * r, 1e8, 0.3);
    s.addBondedInteraction(0, 3, make_double3(-1.96 * r, -0.98 * r, 0.99 * r), make_double3(0, 1, 0), 0.3 * r,
                           1.96 * r, 1e8, 0.3);
    const double L = 1.0;
    std::vector<double> plane(8);
    const double3 po = make_double3(-0.5 * L, -0.5 * L, -0.5 * L);
    for (int z = 0; z < 2; ++z)
        for (int y = 0; y < 2; ++y)
            for (int x = 0; x < 2; ++x) plane[linearIndex3D(make_int3(x, y, z), make_int3(2, 2, 2))] = po.z + z * L;
    std::vector<double3> pnodes = {make_double3(-0.4, -0.4, 0), make_double3(0.4, -0.4, 0), make_double3(0.4, 0.4, 0),
                                   make_double3(-0.4, 0.4, 0)};
    s.addWallMaterial(0.5, 0.5);
    s.addWallGeometry(po, L, make_int3(2, 2, 2), plane, pnodes, std::vector<int3>());
    s.addWall(make_double3(0, 0, 0), make_double3(0, 0, 0), make_double3(0, 0, 0), make_quaternion(1, 0, 0, 0), 0, 0);
    s.solve(make_double3(-0.2, -0.2, -0.05), make_double3(0.2, 0.2, 0.2), make_double3(0, 0, -9.81), 1e-5, 2e-4, 1,
            argc, argv);
    if (s.failures) return 1;
    std::printf("views ok %d\n", s.checks);
    return s.checks > 0 ? 0 : 2;
}
