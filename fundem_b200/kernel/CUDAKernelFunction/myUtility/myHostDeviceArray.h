// Caller-side container of the LSSolver call surface: a host std::vector with
// a device mirror, under the names an app written against the reference's
// LSParticle.h can reach (HostDeviceArray1D<T>, CUDA_CHECK,
// check_cuda_error, debug_dump_device_array).  The library keeps its own
// device state elsewhere; this header serves apps and hooks that keep extra
// per-object arrays.
//
// Design:
//   * the device side is one block with a logical size and a capacity; a
//     request that fits the capacity reuses the block, a larger one replaces
//     it (stream-ordered cudaMallocAsync / cudaFreeAsync on the caller's
//     stream), so repeated host-to-device copies of a list that shrinks and
//     grows again do not churn the allocator;
//   * every CUDA call goes through CUDA_CHECK, which throws std::runtime_error;
//   * the destructor and moves release without checking (the runtime may be
//     shutting down) and never throw.
// Not copyable; movable.
#pragma once
#include <cstddef>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

// Throws std::runtime_error naming the failed call, its source location and
// the runtime's description of the error.
inline void check_cuda_error(cudaError_t result, const char* func, const char* file, int line)
{
    if (result == cudaSuccess) return;
    std::ostringstream msg;
    msg << func << " failed with " << cudaGetErrorName(result) << " (" << cudaGetErrorString(result) << "), "
        << file << " line " << line;
    throw std::runtime_error(msg.str());
}

#define CUDA_CHECK(val) check_cuda_error((val), #val, __FILE__, __LINE__)

#ifndef NDEBUG
#include <iostream>

namespace hda_detail {
template <typename T>
inline void print_element(std::ostream& os, const T& v) { os << v; }
inline void print_element(std::ostream& os, const double3& v) { os << v.x << ' ' << v.y << ' ' << v.z; }
inline void print_element(std::ostream& os, const int3& v) { os << v.x << ' ' << v.y << ' ' << v.z; }
}  // namespace hda_detail

// Debug aid: waits for `stream` (the whole device for stream 0), copies the
// first n elements of a device array back and prints one per line,
// "name[i] value".  Compiled out with NDEBUG.
template <typename T>
void debug_dump_device_array(const T* d_ptr, std::size_t n, const char* name, cudaStream_t stream = 0)
{
    if (n == 0 || d_ptr == nullptr) return;
    CUDA_CHECK(stream == 0 ? cudaDeviceSynchronize() : cudaStreamSynchronize(stream));
    std::vector<T> h(n);
    CUDA_CHECK(cudaMemcpy(h.data(), d_ptr, n * sizeof(T), cudaMemcpyDeviceToHost));
    std::ostringstream out;
    for (std::size_t i = 0; i < n; ++i) {
        out << name << '[' << i << "] ";
        hda_detail::print_element(out, h[i]);
        out << '\n';
    }
    std::cout << out.str() << std::flush;
}
#endif

template <typename T>
struct HostDeviceArray1D
{
public:
    T* d_ptr{nullptr};  // device block (null when nothing is allocated)

private:
    std::vector<T> host_;
    std::size_t dev_count_{0};     // logical device size
    std::size_t dev_capacity_{0};  // elements the block can hold

    void forget() noexcept
    {
        d_ptr = nullptr;
        dev_count_ = 0;
        dev_capacity_ = 0;
    }
    void free_unchecked() noexcept
    {
        if (d_ptr) (void)cudaFree(d_ptr);
        forget();
    }
    // device block of at least n elements, size n; contents undefined
    void reserve_device(std::size_t n, cudaStream_t stream)
    {
        if (n > dev_capacity_ || d_ptr == nullptr) {
            if (d_ptr) CUDA_CHECK(cudaFreeAsync(d_ptr, stream));
            forget();
            if (n > 0) CUDA_CHECK(cudaMallocAsync(reinterpret_cast<void**>(&d_ptr), n * sizeof(T), stream));
            dev_capacity_ = n;
        }
        dev_count_ = n;
    }

public:
    HostDeviceArray1D() = default;
    ~HostDeviceArray1D() { free_unchecked(); }
    HostDeviceArray1D(const HostDeviceArray1D&) = delete;
    HostDeviceArray1D& operator=(const HostDeviceArray1D&) = delete;
    HostDeviceArray1D(HostDeviceArray1D&& other) noexcept
        : d_ptr(std::exchange(other.d_ptr, nullptr)),
          host_(std::move(other.host_)),
          dev_count_(std::exchange(other.dev_count_, 0)),
          dev_capacity_(std::exchange(other.dev_capacity_, 0))
    {
        other.host_.clear();
    }
    HostDeviceArray1D& operator=(HostDeviceArray1D&& other) noexcept
    {
        if (this == &other) return *this;
        free_unchecked();
        d_ptr = std::exchange(other.d_ptr, nullptr);
        dev_count_ = std::exchange(other.dev_count_, 0);
        dev_capacity_ = std::exchange(other.dev_capacity_, 0);
        host_ = std::move(other.host_);
        other.host_.clear();
        return *this;
    }

    // sizes
    std::size_t hostSize() const { return host_.size(); }
    std::size_t deviceSize() const { return dev_count_; }
    double deviceMemoryGB() const { return double(dev_count_ * sizeof(T)) / double(1ull << 30); }

    // device block
    void releaseDevice(cudaStream_t stream)
    {
        T* p = d_ptr;
        forget();
        if (p) CUDA_CHECK(cudaFreeAsync(p, stream));
    }
    void releaseDeviceSync()
    {
        T* p = d_ptr;
        forget();
        if (p) CUDA_CHECK(cudaFree(p));
    }
    // n elements on the device, zeroed unless zeroFill is false (stream-ordered)
    void allocateDevice(std::size_t n, cudaStream_t stream, bool zeroFill = true)
    {
        reserve_device(n, stream);
        if (zeroFill && n > 0) CUDA_CHECK(cudaMemsetAsync(d_ptr, 0, n * sizeof(T), stream));
    }

    // host vector
    void pushHost(const T& value) { host_.push_back(value); }
    // inserts before index; an index at or past the end appends
    void insertHost(std::size_t index, const T& value)
    {
        host_.insert(host_.begin() + static_cast<std::ptrdiff_t>(index < host_.size() ? index : host_.size()), value);
    }
    // an index past the end changes nothing
    void eraseHost(std::size_t index)
    {
        if (index < host_.size()) host_.erase(host_.begin() + static_cast<std::ptrdiff_t>(index));
    }
    void clearHost() { host_.clear(); }
    void reserveHost(std::size_t n) { host_.reserve(n); }
    void resizeHost(std::size_t n) { host_.resize(n); }
    const std::vector<T>& hostRef() const { return host_; }
    void setHost(const std::vector<T>& values) { host_ = values; }

    // transfers (stream-ordered; the host side is complete once the stream
    // reaches the copy)
    // host vector -> device; the device size becomes the host size
    void copyHostToDevice(cudaStream_t stream)
    {
        reserve_device(host_.size(), stream);
        if (!host_.empty())
            CUDA_CHECK(cudaMemcpyAsync(d_ptr, host_.data(), host_.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
    }
    // device -> host vector, resized to the device size
    void copyDeviceToHost(cudaStream_t stream)
    {
        if (d_ptr == nullptr || dev_count_ == 0) return;
        host_.resize(dev_count_);
        CUDA_CHECK(cudaMemcpyAsync(host_.data(), d_ptr, dev_count_ * sizeof(T), cudaMemcpyDeviceToHost, stream));
    }
    // synchronous device -> host copy; returns the refreshed host vector
    std::vector<T> getHostCopy()
    {
        if (d_ptr != nullptr && dev_count_ > 0) {
            host_.resize(dev_count_);
            CUDA_CHECK(cudaMemcpy(host_.data(), d_ptr, dev_count_ * sizeof(T), cudaMemcpyDeviceToHost));
        }
        return host_;
    }
};
