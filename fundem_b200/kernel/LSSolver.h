// LSSolver: the reference's solver class (kernel/LSSolver.h) with the same
// public methods, argument meaning and hook, running the timestep in
// libfundem_b200 through its C ABI (include/fundem_b200.h).  An app written
// against the reference builds unchanged with this directory on its include
// path and links libfundem_b200.so; its addExternalForceTorque override runs
// between the two halves of each step, on the simulation's stream, with the
// device pointers of getLSParticle().
//
// Invalid input is reported on std::cerr and the call is skipped, as in the
// reference.  Differences: solve() writes one particle VTU file per frame
// (centres, velocities, angular velocities; the reference also writes the
// surface mesh and contacts), and addPeriodicBoundarySector is not
// available (the sector periodicity is not part of this library).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "LSParticle.h"
#include "SolidInteraction.h"
#include "VBondedInteraction.h"

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
        }
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
        (void)boundaryNodeConnectivity;  // surface mesh: output only in the reference
        const double I[6] = {inertiaTensor.xx, inertiaTensor.yy, inertiaTensor.zz,
                             inertiaTensor.xy, inertiaTensor.xz, inertiaTensor.yz};
        addGeometry(false, mass, I, gridNodeOrigin, gridNodeSpacing, gridNodeSize, gridNodeSignedDistance,
                    boundaryNodePosition, "addParticleGeometry");
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
        (void)boundaryNodeConnectivity;
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
                                    gridNodeSignedDistance, nodes, "addParticleCluster");
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
        (void)boundaryNodeConnectivity;
        const double I[6] = {0, 0, 0, 0, 0, 0};
        addGeometry(true, 0.0, I, gridNodeOrigin, gridNodeSpacing, gridNodeSize, gridNodeSignedDistance,
                    boundaryNodePosition, "addWallGeometry");
    }

    void addWall(const double3 position, const double3 velocity, const double3 angularVelocity,
                 const quaternion orientation, const int materialID, const int geometryID)
    {
        report(fundem_add_objects(sim_, 1, 1, &position.x, &velocity.x, &angularVelocity.x, &orientation.q0,
                                  &materialID, &geometryID), "addWall");
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
        report(fundem_add_bonds(sim_, 1, &masterObjectID, &slaveObjectID, &bondPoint.x, &bondNormal.x, &radius,
                                &initialLength, &YoungsModulus, &poissonRatio, &tensileStrength, &cohesion,
                                &frictionCoefficient), "addBondedInteraction");
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
        for (size_t i = 0; i < particleGeo_.size(); ++i) nodeBase[i + 1] = nodeBase[i] + geoNodes_[particleGeo_[i]];
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

    // ---------------------------------------------------------------- run
    // the loop of LSSolver::compute* (LSSolver.h:440-467, 1091-1229):
    // numStep = Tmax / dt + 1, iStep = 0 .. numStep inclusive
    void solve(const double3 minDomain, const double3 maxDomain, const double3 gravity, const double timeStep,
               const double maximumTime, const size_t numFrame, const int argc, char** argv)
    {
        (void)argc;
        (void)argv;
        if (!sim_) return;
        if (!(timeStep > 0.0) || !(maximumTime > 0.0) || !(minDomain.x < maxDomain.x) ||
            !(minDomain.y < maxDomain.y) || !(minDomain.z < maxDomain.z)) {
            std::cerr << "[LSSolver] solve: invalid time step, maximum time or domain" << std::endl;
            return;
        }
        phase_ += 1;
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
                    const std::vector<double>& sdf, const std::vector<double3>& nodes, const char* what)
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
        if (!wall) {
            if ((int)geoNodes_.size() <= id) geoNodes_.resize(id + 1, 0);
            geoNodes_[id] = (int)nodes.size();
        }
        return id;
    }

    // one VTU file of particle centres per frame, in <dir>_phase<k>/LSParticle/
    void output(size_t iFrame, size_t iStep, double time)
    {
        const std::string dir = dir_ + "_phase" + std::to_string(phase_);
        const std::string sub = dir + "/LSParticle";
        mkdir(dir.c_str(), 0755);
        mkdir(sub.c_str(), 0755);
        char name[64];
        std::snprintf(name, sizeof(name), "/LSParticle_%04zu.vtu", iFrame);
        LSParticle_.download();
        const std::vector<double3>& x = LSParticle_.positionHostRef();
        const std::vector<double3>& v = LSParticle_.velocityHostRef();
        const std::vector<double3>& w = LSParticle_.angularVelocityHostRef();
        std::ofstream f(sub + name);
        if (!f) {
            std::cerr << "[LSSolver] cannot write " << sub + name << std::endl;
            return;
        }
        f << "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"0.1\">\n<UnstructuredGrid>\n";
        f << "<FieldData><DataArray type=\"Float64\" Name=\"TIME\" NumberOfTuples=\"1\" format=\"ascii\">" << time
          << "</DataArray><DataArray type=\"Int64\" Name=\"STEP\" NumberOfTuples=\"1\" format=\"ascii\">" << iStep
          << "</DataArray></FieldData>\n";
        f << "<Piece NumberOfPoints=\"" << x.size() << "\" NumberOfCells=\"0\">\n<Points>\n"
          << "<DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n";
        f.precision(17);
        for (const double3& p : x) f << p.x << ' ' << p.y << ' ' << p.z << '\n';
        f << "</DataArray>\n</Points>\n<PointData>\n";
        auto vec = [&](const char* nm, const std::vector<double3>& a) {
            f << "<DataArray type=\"Float64\" Name=\"" << nm << "\" NumberOfComponents=\"3\" format=\"ascii\">\n";
            for (const double3& p : a) f << p.x << ' ' << p.y << ' ' << p.z << '\n';
            f << "</DataArray>\n";
        };
        vec("velocity", v);
        vec("angularVelocity", w);
        f << "</PointData>\n<Cells>\n<DataArray type=\"Int32\" Name=\"connectivity\" format=\"ascii\"></DataArray>\n"
          << "<DataArray type=\"Int32\" Name=\"offsets\" format=\"ascii\"></DataArray>\n"
          << "<DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\"></DataArray>\n</Cells>\n"
          << "</Piece>\n</UnstructuredGrid>\n</VTKFile>\n";
    }

    std::string dir_;
    cudaStream_t stream_;
    size_t maxGPUThread_;
    int device_;
    fundem_sim* sim_ = nullptr;
    int phase_ = 0;
    bool perX_ = false, perY_ = false;
    std::vector<int> geoNodes_;     // boundary nodes per particle geometry
    std::vector<int> particleGeo_;  // geometry of each particle
    std::vector<double3> wallVel_, wallAng_;
    LSParticle LSParticle_;
    LSParticle Wall_;
    SolidInteraction LSParticleInteraction_;
    SolidInteraction LSParticleWallInteraction_;
    VBondedInteraction VBondedInteraction_;
};
