// LSParticle view of one object set (particles or walls) of a simulation in
// libfundem_b200: the device pointers and launch shape an
// addExternalForceTorque hook uses (reference: kernel/LSParticle.h:764-777),
// and host copies of the state.  The pointers come from the library
// (fundem_device_view_get) and stay valid until the next solve() re-uploads
// the objects.
#pragma once
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/fundem_b200.h"
#include "CUDAKernelFunction/myUtility/myFileEdit.h"
#include "CUDAKernelFunction/myUtility/myHostDeviceArray.h"
#include "CUDAKernelFunction/myUtility/myMat.h"
#include "CUDAKernelFunction/myUtility/myQua.h"
#include "CUDAKernelFunction/myUtility/myVec.h"

namespace fundem_detail {
inline void check(int status, const char* what)
{
    if (status != FUNDEM_OK)
        throw std::runtime_error(std::string(what) + ": " + fundem_status_string(status));
}
}  // namespace fundem_detail

class LSParticle {
public:
    explicit LSParticle(bool wall) : wall_(wall) {}

    void bind(fundem_sim* sim, size_t maxGPUThread)
    {
        sim_ = sim;
        blockDim_ = maxGPUThread > 0 ? maxGPUThread : 256;
        refresh();
    }

    size_t num_device() const { refresh(); return (size_t)view_.n; }
    const size_t& gridDim() const { refresh(); return gridDim_; }
    const size_t& blockDim() const { return blockDim_; }

    double3* position() { refresh(); return reinterpret_cast<double3*>(view_.pos); }
    double3* velocity() { refresh(); return reinterpret_cast<double3*>(view_.vel); }
    double3* angularVelocity() { refresh(); return reinterpret_cast<double3*>(view_.angvel); }
    double3* force() { refresh(); return reinterpret_cast<double3*>(view_.force); }
    double3* torque() { refresh(); return reinterpret_cast<double3*>(view_.torque); }
    quaternion* orientation() { refresh(); return reinterpret_cast<quaternion*>(view_.quat); }
    int* materialID() { refresh(); return view_.mat; }
    int* geometryID() { refresh(); return view_.geo; }

    // host copies of the current state (waits for the simulation's stream)
    void download()
    {
        int n = 0;
        fundem_detail::check(fundem_num_objects(sim_, wall_, &n), "num_objects");
        pos_.resize(n); vel_.resize(n); angvel_.resize(n); force_.resize(n); torque_.resize(n); q_.resize(n);
        if (n == 0) return;
        fundem_detail::check(fundem_get_objects(sim_, wall_, &pos_[0].x, &vel_[0].x, &angvel_[0].x, &q_[0].q0,
                                                &force_[0].x, &torque_[0].x), "get_objects");
    }
    const std::vector<double3>& positionHostRef() { download(); return pos_; }
    const std::vector<double3>& velocityHostRef() { download(); return vel_; }
    const std::vector<double3>& angularVelocityHostRef() { download(); return angvel_; }
    const std::vector<double3>& forceHostRef() { download(); return force_; }
    const std::vector<double3>& torqueHostRef() { download(); return torque_; }
    const std::vector<quaternion>& orientationHostRef() { download(); return q_; }
    // the copies made by the last download(), without another transfer
    const std::vector<double3>& positionHost() const { return pos_; }
    const std::vector<double3>& velocityHost() const { return vel_; }
    const std::vector<double3>& angularVelocityHost() const { return angvel_; }
    const std::vector<quaternion>& orientationHost() const { return q_; }

private:
    void refresh() const
    {
        if (!sim_) throw std::runtime_error("LSParticle: the solver has not been set up (call solve first)");
        fundem_detail::check(fundem_device_view_get(sim_, wall_, &view_), "device_view_get");
        gridDim_ = ((size_t)view_.n + blockDim_ - 1) / blockDim_;
        if (gridDim_ == 0) gridDim_ = 1;
    }

    fundem_sim* sim_ = nullptr;
    bool wall_;
    mutable fundem_device_view view_{};
    mutable size_t gridDim_ = 1;
    size_t blockDim_ = 256;
    std::vector<double3> pos_, vel_, angvel_, force_, torque_;
    std::vector<quaternion> q_;
};
