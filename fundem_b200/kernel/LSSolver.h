// LSSolver: the reference's solver class (kernel/LSSolver.h) with the same
// public methods, argument meaning and hook, running the timestep in
// libfundem_b200 through its C ABI (include/fundem_b200.h).  An app written
// against the reference builds unchanged with this directory on its include
// path and links libfundem_b200.so; its addExternalForceTorque override runs
// between the two halves of each step, on the simulation's stream, with the
// device pointers of getLSParticle().
//
// Invalid input is reported on std::cerr and the call is skipped, as in the
// reference.  solve() writes the reference's frame files (LSSolver.h:717-744):
// particle and wall surface meshes, particle centres, particle and wall
// contacts and bonds, as VTK XML files (VTUWriter.h).  Contact lists are in
// canonical (node, partner) order, which the reference does not fix.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "LSParticle.h"
#include "SolidInteraction.h"
#include "VBondedInteraction.h"
#include "VTUWriter.h"

class LSSolver {
public:
    LSSolver(const std::string dir = "Problem", cudaStream_t stream = 0, const size_t maxGPUThread = 256,
             const int device = 0)
        : dir_(dir), stream_(stream), maxGPUThread_(maxGPUThread), device_(device), LSParticle_(false),
          Wall_(true), LSParticleInteraction_(FUNDEM_PP), LSParticleWallInteraction_(FUNDEM_PW)
    {
        const int r = fundem_create(&sim_, device, (void*)stream);
        if (r != FUNDEM_OK) {
            std::cerr << "[LSSolver] cannot use CUDA device " << device << ": " << fundem_status_string(r)
                      << std::endl;
            sim_ = nullptr;
            return;
        }
        // every step keeps contact points, normals and energies for the frames
        fundem_set_records(sim_, 1);
    }
    virtual ~LSSolver()
    {
        if (sim_) fundem_destroy(sim_);
    }
    LSSolver(const LSSolver&) = delete;
    LSSolver& operator=(const LSSolver&) = delete;

    // ---------------------------------------------------------------- input
    void addParticleMaterial(const double normalStiffness, const double shearStiffness,
                             const double frictionCoefficient, const double restitutionCoefficient)
    {
        int id = 0;
        report(fundem_add_material(sim_, 0, normalStiffness, shearStiffness, frictionCoefficient,
                                   restitutionCoefficient, &id), "addParticleMaterial");
    }

    void addParticleGeometry(const double mass, const symMatrix inertiaTensor, const double3 gridNodeOrigin,
                             const double gridNodeSpacing, const int3 gridNodeSize,
                             const std::vector<double>& gridNodeSignedDistance,
                             const std::vector<double3>& boundaryNodePosition,
                             const std::vector<int3>& boundaryNodeConnectivity)
    {
        const double I[6] = {inertiaTensor.xx, inertiaTensor.yy, inertiaTensor.zz,
                             inertiaTensor.xy, inertiaTensor.xz, inertiaTensor.yz};
        addGeometry(false, mass, I, gridNodeOrigin, gridNodeSpacing, gridNodeSize, gridNodeSignedDistance,
                    boundaryNodePosition, boundaryNodeConnectivity, "addParticleGeometry");
    }

    void addParticle(const double3 position, const double3 velocity, const double3 angularVelocity,
                     const quaternion orientation, const int materialID, const int geometryID)
    {
        if (geometryID < 0 || geometryID >= (int)geoNodes_.size()) {
            std::cerr << "[LSSolver] addParticle: invalid geometry ID " << geometryID << std::endl;
            return;
        }
        if (report(fundem_add_objects(sim_, 0, 1, &position.x, &velocity.x, &angularVelocity.x, &orientation.q0,
                                      &materialID, &geometryID), "addParticle"))
            particleGeo_.push_back(geometryID);
    }

    // particles of one shape whose mass, centroid and inertia follow from a
    // density; the template is shifted to its centroid and the given
    // positions follow it (LSSolver.h:125-165)
    void addParticleCluster(const std::vector<double3>& position, const std::vector<double3>& velocity,
                            const std::vector<double3>& angularVelocity, const std::vector<quaternion>& orientation,
                            const int materialID, const double density, const double3 gridNodeOrigin,
                            const double gridNodeSpacing, const int3 gridNodeSize,
                            const std::vector<double>& gridNodeSignedDistance,
                            const std::vector<double3>& boundaryNodePosition,
                            const std::vector<int3>& boundaryNodeConnectivity)
    {
        const size_t n = position.size();
        if (velocity.size() != n || angularVelocity.size() != n || orientation.size() != n) {
            std::cerr << "[LSSolver] addParticleCluster: array sizes differ" << std::endl;
            return;
        }
        const int size[3] = {gridNodeSize.x, gridNodeSize.y, gridNodeSize.z};
        double mass = 0.0, c[3] = {0, 0, 0}, I[6] = {0, 0, 0, 0, 0, 0};
        if (!report(fundem_mass_properties(density, &gridNodeOrigin.x, gridNodeSpacing, size,
                                           gridNodeSignedDistance.data(), &mass, c, I), "addParticleCluster"))
            return;
        const double3 cen = make_double3(c[0], c[1], c[2]);
        std::vector<double3> nodes(boundaryNodePosition);
        for (double3& p : nodes) p = p - cen;
        const int geo = addGeometry(false, mass, I, gridNodeOrigin - cen, gridNodeSpacing, gridNodeSize,
                                    gridNodeSignedDistance, nodes, boundaryNodeConnectivity, "addParticleCluster");
        if (geo < 0) return;
        for (size_t i = 0; i < n; ++i)
            addParticle(position[i] + rotateVectorByQuaternion(orientation[i], cen), velocity[i],
                        angularVelocity[i], orientation[i], materialID, geo);
    }

    void addWallMaterial(const double frictionCoefficient, const double restitutionCoefficient)
    {
        int id = 0;
        report(fundem_add_material(sim_, 1, 0.0, 0.0, frictionCoefficient, restitutionCoefficient, &id),
               "addWallMaterial");
    }

    void addWallGeometry(const double3 gridNodeOrigin, const double gridNodeSpacing, const int3 gridNodeSize,
                         const std::vector<double>& gridNodeSignedDistance,
                         const std::vector<double3>& boundaryNodePosition,
                         const std::vector<int3>& boundaryNodeConnectivity)
    {
        const double I[6] = {0, 0, 0, 0, 0, 0};
        addGeometry(true, 0.0, I, gridNodeOrigin, gridNodeSpacing, gridNodeSize, gridNodeSignedDistance,
                    boundaryNodePosition, boundaryNodeConnectivity, "addWallGeometry");
    }

    void addWall(const double3 position, const double3 velocity, const double3 angularVelocity,
                 const quaternion orientation, const int materialID, const int geometryID)
    {
        if (report(fundem_add_objects(sim_, 1, 1, &position.x, &velocity.x, &angularVelocity.x, &orientation.q0,
                                      &materialID, &geometryID), "addWall"))
            wallGeo_.push_back(geometryID);
    }

    void moveLSParticle(const size_t index, const double3 offSet)
    {
        report(fundem_move(sim_, 0, (int)index, &offSet.x), "moveLSParticle");
    }
    void moveWall(const size_t index, const double3 offset)
    {
        report(fundem_move(sim_, 1, (int)index, &offset.x), "moveWall");
    }
    void setFixedVelocityToWall(const size_t index, const double3 velocity)
    {
        wallVel_.resize(std::max(wallVel_.size(), index + 1), make_double3(0, 0, 0));
        wallAng_.resize(wallVel_.size(), make_double3(0, 0, 0));
        wallVel_[index] = velocity;
        report(fundem_set_wall_motion(sim_, (int)index, &wallVel_[index].x, &wallAng_[index].x),
               "setFixedVelocityToWall");
    }
    void setFixedAngularVelocityToWall(const size_t index, const double3 angularVelocity)
    {
        wallVel_.resize(std::max(wallVel_.size(), index + 1), make_double3(0, 0, 0));
        wallAng_.resize(wallVel_.size(), make_double3(0, 0, 0));
        wallAng_[index] = angularVelocity;
        report(fundem_set_wall_motion(sim_, (int)index, &wallVel_[index].x, &wallAng_[index].x),
               "setFixedAngularVelocityToWall");
    }

    void addBondedInteraction(const int masterObjectID, const int slaveObjectID, const double3 bondPoint,
                              const double3 bondNormal, const double radius, const double initialLength,
                              const double YoungsModulus, const double poissonRatio,
                              const double tensileStrength = 0., const double cohesion = 0.,
                              const double frictionCoefficient = 0.)
    {
        if (report(fundem_add_bonds(sim_, 1, &masterObjectID, &slaveObjectID, &bondPoint.x, &bondNormal.x, &radius,
                                    &initialLength, &YoungsModulus, &poissonRatio, &tensileStrength, &cohesion,
                                    &frictionCoefficient), "addBondedInteraction")) {
            bondMaster_.push_back(masterObjectID);
            bondSlave_.push_back(slaveObjectID);
        }
    }

    // one bond per current particle-particle node contact (LSSolver.h:347-380)
    void createBondsFromLSInteractions(const double radius, const double initialLength, const double YoungsModulus,
                                       const double poissonRatio, const double tensileStrength = 0.,
                                       const double cohesion = 0., const double frictionCoefficient = 0.)
    {
        SolidInteraction& I = LSParticleInteraction_;
        I.download();
        const std::vector<int> node = I.masterIDHostRef();
        const std::vector<int> slave = I.slaveIDHostRef();
        const std::vector<double3> point = I.contactPointHostRef();
        const std::vector<double3> normal = I.contactNormalHostRef();
        std::vector<int> nodeBase(particleGeo_.size() + 1, 0);
        for (size_t i = 0; i < particleGeo_.size(); ++i)
            nodeBase[i + 1] = nodeBase[i] + (int)geoNodes_[particleGeo_[i]].size();
        for (size_t k = 0; k < node.size(); ++k) {
            const int i = (int)(std::upper_bound(nodeBase.begin(), nodeBase.end(), node[k]) - nodeBase.begin()) - 1;
            addBondedInteraction(i, slave[k], point[k], normal[k], radius, initialLength, YoungsModulus,
                                 poissonRatio, tensileStrength, cohesion, frictionCoefficient);
        }
    }

    void addPeriodicBoundaryXD() { perX_ = true; report(fundem_set_periodic(sim_, perX_, perY_), "periodic"); }
    void addPeriodicBoundaryYD() { perY_ = true; report(fundem_set_periodic(sim_, perX_, perY_), "periodic"); }
    void addPeriodicBoundarySector() { report(fundem_set_periodic_sector(sim_, 1), "addPeriodicBoundarySector"); }
    void removePeriodicBoundary()
    {
        perX_ = perY_ = false;
        report(fundem_set_periodic(sim_, 0, 0), "removePeriodicBoundary");
        report(fundem_set_periodic_sector(sim_, 0), "removePeriodicBoundary");
    }

    // Not in the reference: physical = true inverts every particle inertia
    // that is not singular relative to its own scale, so millimetre bodies
    // turn under contact torques; false (default) keeps inverse()'s
    // |det| < 1e-30 -> zero rule (myMat.h:163-194).  Applies from the next
    // solve().
    void usePhysicalInertia(const bool physical)
    {
        report(fundem_set_inertia_mode(sim_, physical ? FUNDEM_INERTIA_PHYSICAL : FUNDEM_INERTIA_REFERENCE),
               "usePhysicalInertia");
    }

    // ---------------------------------------------------------------- run
    // the loop of LSSolver::compute* (LSSolver.h:440-467, 1091-1229):
    // numStep = Tmax / dt + 1, iStep = 0 .. numStep inclusive
    void solve(const double3 minDomain, const double3 maxDomain, const double3 gravity, const double timeStep,
               const double maximumTime, const size_t numFrame, const int argc, char** argv)
    {
        if (!sim_) return;
        if (!(timeStep > 0.0) || !(maximumTime > 0.0) || !(minDomain.x < maxDomain.x) ||
            !(minDomain.y < maxDomain.y) || !(minDomain.z < maxDomain.z)) {
            std::cerr << "[LSSolver] solve: invalid time step, maximum time or domain" << std::endl;
            return;
        }
        phase_ += 1;
        resolveDir(argc > 0 ? argv[0] : nullptr);
        clearFrames();
        if (!report(fundem_setup(sim_, &minDomain.x, &maxDomain.x), "solve: setup")) return;
        LSParticle_.bind(sim_, maxGPUThread_);
        Wall_.bind(sim_, maxGPUThread_);
        LSParticleInteraction_.bind(sim_);
        LSParticleWallInteraction_.bind(sim_);
        VBondedInteraction_.bind(sim_);
        if (!report(fundem_detect(sim_), "solve: detection")) return;
        const size_t numStep = size_t(maximumTime / timeStep) + 1;
        size_t frameInterval = numStep;
        if (numFrame > 0) frameInterval = numStep / numFrame;
        if (frameInterval < 1) frameInterval = 1;
        size_t iStep = 0, iFrame = 0;
        double time = 0.0;
        output(iFrame, iStep, time);
        while (iStep <= numStep) {
            if (!report(fundem_step_begin(sim_, &gravity.x, timeStep), "solve: step")) return;
            addExternalForceTorque(time);
            if (!report(fundem_step_end(sim_, &gravity.x, timeStep), "solve: step")) return;
            iStep += 1;
            time += timeStep;
            if (iStep % frameInterval == 0) output(++iFrame, iStep, time);
        }
        output(++iFrame, iStep, time);
        report(fundem_sync(sim_), "solve");
    }

protected:
    virtual void addExternalForceTorque(const double time) { (void)time; }

    LSParticle& getLSParticle() { return LSParticle_; }
    LSParticle& getWall() { return Wall_; }
    SolidInteraction& getLSParticleInteraction() { return LSParticleInteraction_; }
    SolidInteraction& getLSParticleWallInteraction() { return LSParticleWallInteraction_; }
    VBondedInteraction& getLSParticleBondedInteraction() { return VBondedInteraction_; }

    // the simulation behind this solver, for calls the class does not wrap
    fundem_sim* simulation() { return sim_; }

private:
    bool report(int status, const char* what)
    {
        if (status == FUNDEM_OK) return true;
        std::cerr << "[LSSolver] " << what << ": " << fundem_status_string(status);
        if (sim_) {
            const char* detail = fundem_last_error(sim_);
            if (detail && *detail) std::cerr << " (" << detail << ")";
        }
        std::cerr << std::endl;
        return false;
    }

    int addGeometry(bool wall, double mass, const double I[6], double3 origin, double spacing, int3 size,
                    const std::vector<double>& sdf, const std::vector<double3>& nodes,
                    const std::vector<int3>& triangles, const char* what)
    {
        const int sz[3] = {size.x, size.y, size.z};
        if ((long long)sdf.size() != (long long)size.x * size.y * size.z) {
            std::cerr << "[LSSolver] " << what << ": signed distance array does not match the grid size" << std::endl;
            return -1;
        }
        int id = -1;
        if (!report(fundem_add_geometry(sim_, wall, mass, I, &origin.x, spacing, sz, sdf.data(), (int)nodes.size(),
                                        nodes.empty() ? nullptr : &nodes[0].x, &id), what))
            return -1;
        // body-frame nodes and triangles of the template, for the frames
        std::vector<std::vector<double3>>& N = wall ? wallGeoNodes_ : geoNodes_;
        std::vector<std::vector<int3>>& T = wall ? wallGeoTris_ : geoTris_;
        if ((int)N.size() <= id) { N.resize(id + 1); T.resize(id + 1); }
        N[id] = nodes;
        T[id] = triangles;
        return id;
    }

    // a relative output name lives beside the executable: under the nearest
    // ancestor directory named "build", else in the executable's own
    // directory (LSSolver.h:615-644); an absolute name is kept
    void resolveDir(const char* exe)
    {
        namespace fs = std::filesystem;
        const fs::path name(dir_);
        if (name.is_absolute()) return;
        if (exe == nullptr) {
            dir_ = (fs::current_path() / name).string();
            return;
        }
        const fs::path here = fs::weakly_canonical(fs::absolute(fs::path(exe))).parent_path();
        fs::path base = here;
        for (fs::path d = here; !d.empty(); d = d.parent_path()) {
            if (d.filename() == "build") {
                base = d;
                break;
            }
            if (d == d.parent_path()) break;
        }
        dir_ = (base / name).string();
    }

    // frames of an earlier run of the same phase are removed before the
    // first frame is written (LSSolver.h:678-690)
    void clearFrames()
    {
        namespace fs = std::filesystem;
        const std::string dir = dir_ + "_phase" + std::to_string(phase_);
        for (const char* sub : {"/LSParticle", "/LSParticleInteraction", "/Wall", "/LSParticle-WallInteraction"}) {
            std::error_code ec;
            const fs::path d(dir + sub);
            if (!fs::is_directory(d, ec)) continue;
            for (const fs::directory_entry& e : fs::directory_iterator(d, ec))
                if (e.is_regular_file(ec) && e.path().extension() == ".vtu") fs::remove(e.path(), ec);
        }
    }

    // the frame files of LSSolver::output (LSSolver.h:717-744), in
    // <dir>_phase<k>/LSParticle, LSParticleInteraction, Wall and
    // LSParticle-WallInteraction
    void output(size_t iFrame, size_t iStep, double time)
    {
        const std::string dir = dir_ + "_phase" + std::to_string(phase_);
        const std::string dP = dir + "/LSParticle", dPI = dir + "/LSParticleInteraction", dW = dir + "/Wall",
                          dWI = dir + "/LSParticle-WallInteraction";
        for (const std::string& d : {dir, dP, dPI, dW, dWI}) mkdir(d.c_str(), 0755);
        char num[16];
        std::snprintf(num, sizeof(num), "_%04zu.vtu", iFrame);
        bool ok = true;
        LSParticle_.download();
        Wall_.download();
        ok &= writeMesh(dP + "/LSObjectMesh" + num, LSParticle_, particleGeo_, geoNodes_, geoTris_, time, iStep);
        ok &= writeCentres(dP + "/Particle" + num, time, iStep);
        ok &= writeContacts(dPI + "/LSInteraction" + num, FUNDEM_PP, time, iStep);
        ok &= writeBonds(dPI + "/VBondedInteraction" + num, time, iStep);
        ok &= writeMesh(dW + "/LSObjectMesh" + num, Wall_, wallGeo_, wallGeoNodes_, wallGeoTris_, time, iStep);
        ok &= writeContacts(dWI + "/LSInteraction" + num, FUNDEM_PW, time, iStep);
        if (!ok) std::cerr << "[LSSolver] cannot write the frame files in " << dir << std::endl;
    }

    static void put3(std::vector<float>& a, double3 v)
    {
        a.push_back(float(v.x));
        a.push_back(float(v.y));
        a.push_back(float(v.z));
    }

    // surface meshes of a set: nodes in the world frame with the body's
    // velocity there, triangles, and the body index of each node
    bool writeMesh(const std::string& file, const LSParticle& set, const std::vector<int>& objGeo,
                   const std::vector<std::vector<double3>>& nodes, const std::vector<std::vector<int3>>& tris,
                   double time, size_t step)
    {
        const std::vector<double3>& x = set.positionHost();
        if (x.empty()) return true;
        const std::vector<double3>& v = set.velocityHost();
        const std::vector<double3>& w = set.angularVelocityHost();
        const std::vector<quaternion>& q = set.orientationHost();
        std::vector<float> points, vel;
        std::vector<int32_t> id, conn, offs;
        std::vector<uint8_t> types;
        int32_t base = 0;
        for (size_t i = 0; i < x.size() && i < objGeo.size(); ++i) {
            const int g = objGeo[i];
            for (const double3& b : nodes[g]) {
                const double3 p = x[i] + rotateVectorByQuaternion(q[i], b);
                put3(points, p);
                put3(vel, v[i] + cross(w[i], p - x[i]));
                id.push_back((int32_t)i);
            }
            for (const int3& t : tris[g]) {
                conn.push_back(base + t.x);
                conn.push_back(base + t.y);
                conn.push_back(base + t.z);
                offs.push_back((int32_t)conn.size());
                types.push_back(5);  // triangle
            }
            base += (int32_t)nodes[g].size();
        }
        return fundem_vtu::write(file, time, (long long)step, points, conn, offs, types,
                                 {fundem_vtu::array("particleID", 1, id), fundem_vtu::array("velocity", 3, vel)});
    }

    bool writeCentres(const std::string& file, double time, size_t step)
    {
        const std::vector<double3>& x = LSParticle_.positionHost();
        if (x.empty()) return true;
        const std::vector<double3>& v = LSParticle_.velocityHost();
        const std::vector<double3>& w = LSParticle_.angularVelocityHost();
        const std::vector<quaternion>& q = LSParticle_.orientationHost();
        std::vector<float> points, vel, ang, ori;
        for (size_t i = 0; i < x.size(); ++i) {
            put3(points, x[i]);
            put3(vel, v[i]);
            put3(ang, w[i]);
            for (double c : {q[i].q0, q[i].q1, q[i].q2, q[i].q3}) ori.push_back(float(c));
        }
        return fundem_vtu::write(file, time, (long long)step, points, {}, {}, {},
                                 {fundem_vtu::array("velocity", 3, vel), fundem_vtu::array("angularVelocity", 3, ang),
                                  fundem_vtu::array("orientation", 4, ori)});
    }

    // node contacts of one list as vertices: point, normal, direction of the
    // sliding spring and the two elastic energies
    bool writeContacts(const std::string& file, int kind, double time, size_t step)
    {
        long long n = 0;
        if (!report(fundem_num_contacts(sim_, kind, &n), "output")) return false;
        std::vector<int> node(n), partner(n);
        std::vector<double> point(3 * n), normal(3 * n), overlap(n), spring(3 * n), en(n), es(n);
        if (n > 0 && !report(fundem_get_contacts(sim_, kind, node.data(), partner.data(), point.data(), normal.data(),
                                                 overlap.data(), spring.data(), en.data(), es.data()), "output"))
            return false;
        std::vector<float> pts, nrm, dir, fen, fes;
        std::vector<int32_t> conn, offs;
        std::vector<uint8_t> types;
        for (long long k = 0; k < n; ++k) {
            put3(pts, make_double3(point[3 * k], point[3 * k + 1], point[3 * k + 2]));
            put3(nrm, make_double3(normal[3 * k], normal[3 * k + 1], normal[3 * k + 2]));
            put3(dir, normalize(make_double3(spring[3 * k], spring[3 * k + 1], spring[3 * k + 2])));
            fen.push_back(float(en[k]));
            fes.push_back(float(es[k]));
            conn.push_back((int32_t)k);
            offs.push_back((int32_t)k + 1);
            types.push_back(1);  // vertex
        }
        return fundem_vtu::write(file, time, (long long)step, pts, conn, offs, types,
                                 {fundem_vtu::array("contactNormal", 3, nrm), fundem_vtu::array("slidingDirection", 3, dir),
                                  fundem_vtu::array("normalElasticEnergy", 1, fen),
                                  fundem_vtu::array("slidingElasticEnergy", 1, fes)});
    }

    bool writeBonds(const std::string& file, double time, size_t step)
    {
        int n = 0;
        if (!report(fundem_num_bonds(sim_, &n), "output")) return false;
        if (n == 0) return true;
        std::vector<int> act(n);
        std::vector<double> point(3 * n), e(6 * n);
        if (!report(fundem_get_bonds(sim_, act.data(), point.data(), e.data()), "output")) return false;
        std::vector<float> pts;
        std::vector<float> f[6];
        std::vector<int32_t> conn, offs, mid, sid, a32;
        std::vector<uint8_t> types;
        for (int k = 0; k < n; ++k) {
            put3(pts, make_double3(point[3 * k], point[3 * k + 1], point[3 * k + 2]));
            for (int c = 0; c < 6; ++c) f[c].push_back(float(e[6 * k + c]));
            mid.push_back(k < (int)bondMaster_.size() ? bondMaster_[k] : -1);
            sid.push_back(k < (int)bondSlave_.size() ? bondSlave_[k] : -1);
            a32.push_back(act[k]);
            conn.push_back(k);
            offs.push_back(k + 1);
            types.push_back(1);
        }
        return fundem_vtu::write(
            file, time, (long long)step, pts, conn, offs, types,
            {fundem_vtu::array("masterObjectID", 1, mid), fundem_vtu::array("slaveObjectID", 1, sid),
             fundem_vtu::array("activated", 1, a32), fundem_vtu::array("normalElasticEnergy", 1, f[0]),
             fundem_vtu::array("shearElasticEnergy", 1, f[1]), fundem_vtu::array("bendingElasticEnergy", 1, f[2]),
             fundem_vtu::array("torsionElasticEnergy", 1, f[3]), fundem_vtu::array("maxNormalStress", 1, f[4]),
             fundem_vtu::array("maxShearStress", 1, f[5])});
    }

    std::string dir_;
    cudaStream_t stream_;
    size_t maxGPUThread_;
    int device_;
    fundem_sim* sim_ = nullptr;
    int phase_ = 0;
    bool perX_ = false, perY_ = false;
    std::vector<std::vector<double3>> geoNodes_, wallGeoNodes_;  // body-frame nodes per geometry
    std::vector<std::vector<int3>> geoTris_, wallGeoTris_;       // surface triangles per geometry
    std::vector<int> particleGeo_, wallGeo_;                      // geometry of each particle and wall
    std::vector<int> bondMaster_, bondSlave_;                     // bodies of each bond
    std::vector<double3> wallVel_, wallAng_;
    LSParticle LSParticle_;
    LSParticle Wall_;
    SolidInteraction LSParticleInteraction_;
    SolidInteraction LSParticleWallInteraction_;
    VBondedInteraction VBondedInteraction_;
};
