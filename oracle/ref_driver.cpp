// ref_driver.cpp -- runs the UNMODIFIED reference (FunDEM's LSSolver and its
// CUDA kernels, compiled from the reference sources by oracle/Makefile) on a
// scenario file and dumps per-step state, contact lists and bond state.
//
// TEST INFRASTRUCTURE ONLY: this program is how the oracle and the CUDA path
// are pinned to the reference.  It is built into oracle/_ref/ (never
// committed) and runs on a GPU machine; its dumps are reduced to small
// fixtures under tests/golden/ by tests/golden/make_fixtures.py.
//
// Scenario format: see fundem_b200/scenario.py (write_reference_scenario).
// The solver is driven only through the reference's public API
// (LSSolver.h:14-467) plus the protected hook addExternalForceTorque
// (LSSolver.h:588) and getters (:590-598).  Ghost contact lists have no
// getter, so the private members are opened for reading below.
#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <set>
#include <string>
#include <vector>
#include <filesystem>
#include <sstream>
#include <iomanip>
#include <random>
#include <memory>
#include <functional>
#include <unordered_map>
#include <cuda_runtime.h>

#define private public
#define protected public
#include "kernel/LSSolver.h"
#undef private
#undef protected

namespace {

struct Reader {
    std::vector<char> buf;
    size_t pos = 0;
    explicit Reader(const std::string& path)
    {
        std::ifstream f(path, std::ios::binary);
        if (!f) throw std::runtime_error("cannot open " + path);
        buf.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
    }
    template <typename T> T get()
    {
        if (pos + sizeof(T) > buf.size()) throw std::runtime_error("scenario truncated");
        T v;
        std::memcpy(&v, buf.data() + pos, sizeof(T));
        pos += sizeof(T);
        return v;
    }
    double3 d3() { double x = get<double>(), y = get<double>(), z = get<double>(); return make_double3(x, y, z); }
    int3 i3() { int x = get<int32_t>(), y = get<int32_t>(), z = get<int32_t>(); return make_int3(x, y, z); }
};

struct Writer {
    std::ofstream f;
    explicit Writer(const std::string& path) : f(path, std::ios::binary) {}
    template <typename T> void put(const T& v) { f.write(reinterpret_cast<const char*>(&v), sizeof(T)); }
    template <typename T> void arr(const std::vector<T>& v) { if (!v.empty()) f.write(reinterpret_cast<const char*>(v.data()), sizeof(T) * v.size()); }
};

template <typename T> std::vector<T> fetch(const T* d, size_t n)
{
    std::vector<T> h(n);
    if (n > 0 && d) cudaMemcpy(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost);
    return h;
}

void dump_contacts(Writer& w, SolidInteraction& c)
{
    const size_t n = c.numPair_device();
    w.put<int64_t>((int64_t)n);
    w.arr(fetch(c.masterID(), n));
    w.arr(fetch(c.slaveID(), n));
    w.arr(fetch(c.contactPoint(), n));
    w.arr(fetch(c.contactNormal(), n));
    w.arr(fetch(c.contactOverlap(), n));
    w.arr(fetch(c.slidingSpring(), n));
    w.arr(fetch(c.normalElasticEnergy(), n));
    w.arr(fetch(c.slidingElasticEnergy(), n));
}

void dump_empty_contacts(Writer& w) { w.put<int64_t>(0); }

class DumpSolver : public LSSolver {
public:
    DumpSolver(const std::string& dir, const std::string& out) : LSSolver(dir), out_(out) {}
    std::set<int64_t> dumpSteps;
    int64_t step = 0;
    bool timingOnly = false;
    bool exitAfterWindow = false;  // timing mode: stop once the window is measured
    // timing window: wall time between the hooks of steps windowFrom and
    // windowTo, after a device synchronisation at each end.  No output frame
    // falls inside when windowTo is below the last step.
    int64_t windowFrom = 0, windowTo = 0;
    std::chrono::steady_clock::time_point tFrom, tTo;
    std::string out_;

    void addExternalForceTorque(const double time) override
    {
        step += 1;
        if (timingOnly) {
            if (step == windowFrom || step == windowTo) {
                cudaDeviceSynchronize();
                (step == windowFrom ? tFrom : tTo) = std::chrono::steady_clock::now();
            }
            if (exitAfterWindow && step == windowTo && windowTo > windowFrom) {
                // the window is all a timing run needs: report it and leave
                // before the remaining steps and the closing frame output
                const double w = std::chrono::duration<double>(tTo - tFrom).count();
                const cudaError_t err = cudaGetLastError();
                std::ofstream meta(out_ + "/meta.txt");
                meta << "steps " << step << "\n";
                meta << "cuda_status " << cudaGetErrorString(err) << "\n";
                meta << "window_steps " << (windowTo - windowFrom) << "\n";
                meta << "window_seconds " << w << "\n";
                meta.close();
                std::cout << "ref_driver: window " << windowFrom << ".." << windowTo << ": "
                          << 1e3 * w / double(windowTo - windowFrom) << " ms/step" << std::endl;
                std::_Exit(err == cudaSuccess ? 0 : 1);
            }
            return;
        }
        if (step == 1) dumpGeometry();
        if (!dumpSteps.count(step)) return;
        cudaStreamSynchronize(0);
        cudaDeviceSynchronize();
        std::ostringstream name;
        name << out_ << "/dump_" << std::setw(6) << std::setfill('0') << step << ".bin";
        Writer w(name.str());
        LSParticle& P = getLSParticle();
        LSParticle& W = getWall();
        const size_t nP = P.num_device(), nW = W.num_device();
        w.put<int64_t>(step);
        w.put<double>(time);
        w.put<int32_t>((int32_t)nP);
        w.put<int32_t>((int32_t)nW);
        w.arr(fetch(P.position(), nP));
        w.arr(fetch(P.velocity(), nP));
        w.arr(fetch(P.angularVelocity(), nP));
        w.arr(fetch(P.orientation(), nP));
        w.arr(fetch(P.force(), nP));
        w.arr(fetch(P.torque(), nP));
        w.arr(fetch(W.position(), nW));
        w.arr(fetch(W.orientation(), nW));
        dump_contacts(w, getLSParticleInteraction());
        dump_contacts(w, getLSParticleWallInteraction());
        PeriodicBoundaryXY2D& pb = PeriodicBoundaryXY2D_;
        if (pb.ativateXFlag_) dump_contacts(w, pb.X_.ghostSolidInteraction_); else dump_empty_contacts(w);
        if (pb.ativateYFlag_) dump_contacts(w, pb.Y_.ghostSolidInteraction_); else dump_empty_contacts(w);
        if (pb.ativateXFlag_ && pb.ativateYFlag_) dump_contacts(w, pb.XY_.ghostSolidInteraction_); else dump_empty_contacts(w);
        VBondedInteraction& B = getLSParticleBondedInteraction();
        const size_t nB = B.numPair_device();
        w.put<int64_t>((int64_t)nB);
        w.arr(fetch(B.activated(), nB));
        w.arr(fetch(B.centerPoint(), nB));
        w.arr(fetch(B.Un(), nB));
        w.arr(fetch(B.Us(), nB));
        w.arr(fetch(B.Ub(), nB));
        w.arr(fetch(B.Ut(), nB));
        w.arr(fetch(B.maxNormalStress(), nB));
        w.arr(fetch(B.maxShearStress(), nB));
        // the sector images' lists, after the bonds, only when sector periodicity is on
        PeriodicBoundarySector& ps = PeriodicBoundarySector_;
        if (ps.ativateFlag_) {
            dump_contacts(w, ps.R90_.ghostSolidInteraction_);
            dump_contacts(w, ps.R180_.ghostSolidInteraction_);
            dump_contacts(w, ps.R270_.ghostSolidInteraction_);
        }
    }

    void dumpGeometry()
    {
        cudaDeviceSynchronize();
        Writer w(out_ + "/geometry.bin");
        geometryInfo& g = getLSParticle().geometryInfo_;
        const size_t n = g.num();
        w.put<int32_t>((int32_t)n);
        w.arr(fetch(g.radius(), n));
        w.arr(fetch(g.inverseMass(), n));
        w.arr(fetch(g.inertiaTensor(), n));
        w.arr(fetch(g.inverseInertiaTensor(), n));
        w.arr(fetch(g.gridNodeOrigin(), n));
        const size_t nn = g.boundaryNodePositionHostRef().size();
        w.put<int64_t>((int64_t)nn);
        w.arr(fetch(g.boundaryNodePosition(), nn));
        LSParticle& P = getLSParticle();
        const size_t nP = P.num_device();
        w.put<int32_t>((int32_t)nP);
        // positions as uploaded (after the addParticleCluster centroid offset)
        w.arr(P.positionHostRef());
        const spatialGrid& sg = P.spatialGrid_;
        w.put(sg.minimumBoundary()); w.put(sg.maximumBoundary()); w.put(sg.inverseCellSize()); w.put(sg.size3D());
    }
};

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 3) {
        std::cerr << "usage: ref_driver scenario.bin outdir [timing [from to [exit]]]\n";
        return 2;
    }
    const std::string scen = argv[1], out = argv[2];
    const bool timing = (argc > 3 && std::string(argv[3]) == "timing");
    std::filesystem::create_directories(out);
    Reader r(scen);
    if (r.get<uint32_t>() != 0x43534446u) { std::cerr << "bad magic\n"; return 2; }
    const uint32_t version = r.get<uint32_t>();
    if (version != 1) { std::cerr << "bad version\n"; return 2; }
    const double3 minD = r.d3(), maxD = r.d3(), g = r.d3();
    const double dt = r.get<double>();
    const int64_t nSteps = r.get<int64_t>();
    const int32_t perX = r.get<int32_t>(), perY = r.get<int32_t>();
    DumpSolver s(out + "/vtu", out);
    s.timingOnly = timing;
    if (timing && argc > 5) {
        s.windowFrom = std::atoll(argv[4]);
        s.windowTo = std::atoll(argv[5]);
        s.exitAfterWindow = argc > 6 && std::string(argv[6]) == "exit";
    }
    const int32_t nDump = r.get<int32_t>();
    for (int i = 0; i < nDump; ++i) s.dumpSteps.insert(r.get<int32_t>());

    const int32_t nMatP = r.get<int32_t>();
    for (int i = 0; i < nMatP; ++i) {
        double kn = r.get<double>(), ks = r.get<double>(), mu = r.get<double>(), e = r.get<double>();
        s.addParticleMaterial(kn, ks, mu, e);
    }
    const int32_t nMatW = r.get<int32_t>();
    for (int i = 0; i < nMatW; ++i) {
        double mu = r.get<double>(), e = r.get<double>();
        s.addWallMaterial(mu, e);
    }
    struct Geo {
        int mode; double mass, density; symMatrix I; double3 origin; double h; int3 size;
        std::vector<double> sdf; std::vector<double3> nodes; std::vector<int3> tris;
    };
    auto readGeo = [&](bool particle) {
        Geo G;
        G.mode = particle ? r.get<int32_t>() : 0;
        if (particle) {
            G.mass = r.get<double>();
            double I[6];
            for (double& v : I) v = r.get<double>();
            G.I = make_symMatrix(I[0], I[1], I[2], I[3], I[4], I[5]);
            G.density = r.get<double>();
        }
        G.origin = r.d3();
        G.h = r.get<double>();
        G.size = r.i3();
        const size_t ns = (size_t)G.size.x * G.size.y * G.size.z;
        G.sdf.resize(ns);
        for (auto& v : G.sdf) v = r.get<double>();
        const int32_t nn = r.get<int32_t>();
        G.nodes.resize(nn);
        for (auto& v : G.nodes) v = r.d3();
        const int32_t nt = r.get<int32_t>();
        G.tris.resize(nt);
        for (auto& v : G.tris) v = r.i3();
        return G;
    };
    const int32_t nGeoP = r.get<int32_t>();
    std::vector<Geo> geoP;
    for (int i = 0; i < nGeoP; ++i) geoP.push_back(readGeo(true));
    const int32_t nGeoW = r.get<int32_t>();
    for (int i = 0; i < nGeoW; ++i) {
        Geo G = readGeo(false);
        s.addWallGeometry(G.origin, G.h, G.size, G.sdf, G.nodes, G.tris);
    }
    struct Obj { double3 p, v, w; quaternion q; int mat, geo; };
    auto readObj = [&]() {
        Obj o;
        o.p = r.d3(); o.v = r.d3(); o.w = r.d3();
        double q0 = r.get<double>(), q1 = r.get<double>(), q2 = r.get<double>(), q3 = r.get<double>();
        o.q = make_quaternion(q0, q1, q2, q3);
        o.mat = r.get<int32_t>(); o.geo = r.get<int32_t>();
        return o;
    };
    const int32_t nP = r.get<int32_t>();
    std::vector<Obj> parts;
    for (int i = 0; i < nP; ++i) parts.push_back(readObj());
    // Geometries with mode 0 go in through addParticleGeometry (explicit mass
    // and inertia).  Mode-1 geometries go in through addParticleCluster, which
    // computes mass properties from the SDF; the scenario writer orders the
    // particles so that each such geometry's particles are contiguous and the
    // geometries appear in first-use order.
    {
        bool anyCluster = false;
        for (const Geo& G : geoP) anyCluster = anyCluster || (G.mode == 1);
        if (!anyCluster) {
            for (const Geo& G : geoP)
                s.addParticleGeometry(G.mass, G.I, G.origin, G.h, G.size, G.sdf, G.nodes, G.tris);
            for (const Obj& o : parts) s.addParticle(o.p, o.v, o.w, o.q, o.mat, o.geo);
        } else {
            // particles arrive grouped by geometry, geometries in order 0, 1, ...
            size_t i = 0;
            for (int gid = 0; gid < nGeoP; ++gid) {
                const Geo& G = geoP[gid];
                size_t j = i;
                while (j < parts.size() && parts[j].geo == gid) ++j;
                if (G.mode == 0) {
                    s.addParticleGeometry(G.mass, G.I, G.origin, G.h, G.size, G.sdf, G.nodes, G.tris);
                    for (size_t k = i; k < j; ++k)
                        s.addParticle(parts[k].p, parts[k].v, parts[k].w, parts[k].q, parts[k].mat, gid);
                } else {
                    std::vector<double3> p, v, w;
                    std::vector<quaternion> q;
                    for (size_t k = i; k < j; ++k) { p.push_back(parts[k].p); v.push_back(parts[k].v); w.push_back(parts[k].w); q.push_back(parts[k].q); }
                    const int mat = (j > i) ? parts[i].mat : 0;
                    s.addParticleCluster(p, v, w, q, mat, G.density, G.origin, G.h, G.size, G.sdf, G.nodes, G.tris);
                }
                i = j;
            }
            if (i != parts.size()) { std::cerr << "particles not grouped by geometry\n"; return 2; }
        }
    }
    const int32_t nW = r.get<int32_t>();
    for (int i = 0; i < nW; ++i) {
        Obj o = readObj();
        s.addWall(o.p, o.v, o.w, o.q, o.mat, o.geo);
    }
    const int32_t nWallVel = r.get<int32_t>();
    for (int i = 0; i < nWallVel; ++i) {
        const int32_t idx = r.get<int32_t>();
        const double3 v = r.d3(), w = r.d3();
        s.setFixedVelocityToWall(idx, v);
        s.setFixedAngularVelocityToWall(idx, w);
    }
    const int32_t nB = r.get<int32_t>();
    for (int i = 0; i < nB; ++i) {
        const int32_t m = r.get<int32_t>(), sl = r.get<int32_t>();
        const double3 pt = r.d3(), nm = r.d3();
        const double R = r.get<double>(), L0 = r.get<double>(), E = r.get<double>(), nu = r.get<double>();
        const double ts = r.get<double>(), coh = r.get<double>(), mu = r.get<double>();
        s.addBondedInteraction(m, sl, pt, nm, R, L0, E, nu, ts, coh, mu);
    }
    if (perX & 1) s.addPeriodicBoundaryXD();
    if (perX & 2) s.addPeriodicBoundarySector();
    if (perY) s.addPeriodicBoundaryYD();

    // numStep = size_t(Tmax/dt) + 1 and the loop runs numStep + 1 times
    // (LSSolver.h:456, 1097): Tmax = (nSteps - 2 + 0.5) dt gives nSteps.
    const double Tmax = (double(nSteps) - 1.5) * dt;
    auto t0 = std::chrono::steady_clock::now();
    s.solve(minD, maxD, g, dt, Tmax, 1, argc, argv);
    cudaDeviceSynchronize();
    auto t1 = std::chrono::steady_clock::now();
    std::ofstream meta(out + "/meta.txt");
    meta << "steps " << s.step << "\n";
    meta << "wall_seconds " << std::chrono::duration<double>(t1 - t0).count() << "\n";
    cudaError_t err = cudaGetLastError();
    meta << "cuda_status " << cudaGetErrorString(err) << "\n";
    if (s.windowTo > s.windowFrom && s.step >= s.windowTo) {
        const double w = std::chrono::duration<double>(s.tTo - s.tFrom).count();
        meta << "window_steps " << (s.windowTo - s.windowFrom) << "\n";
        meta << "window_seconds " << w << "\n";
        std::cout << "ref_driver: window " << s.windowFrom << ".." << s.windowTo << ": "
                  << 1e3 * w / double(s.windowTo - s.windowFrom) << " ms/step" << std::endl;
    }
    std::cout << "ref_driver: " << s.step << " steps, " << std::chrono::duration<double>(t1 - t0).count()
              << " s, " << cudaGetErrorString(err) << std::endl;
    return err == cudaSuccess ? 0 : 1;
}
