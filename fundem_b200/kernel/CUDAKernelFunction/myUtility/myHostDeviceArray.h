// HostDeviceArray1D<T>, CUDA_CHECK and debug_dump_device_array with the names,
// members and behaviour of the reference's kernel/CUDAKernelFunction/
// myUtility/myHostDeviceArray.h, which LSParticle.h includes, so hooks and
// apps that keep their own per-object arrays this way build unchanged.  The
// library itself keeps its device state elsewhere; this is a container for
// the caller.
//
// A host vector and a device copy: the device side is allocated
// stream-ordered (cudaMallocAsync / cudaFreeAsync on the given stream, or
// cudaFree for the synchronous release and on destruction), copies are
// stream-ordered, and a host-to-device copy reallocates when the sizes
// differ.  Not copyable; movable.
#pragma once
#include <cstddef>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

inline void check_cuda_error(cudaError_t result, const char* func, const char* file, int line)
{
    if (result == cudaSuccess) return;
    throw std::runtime_error(std::string("CUDA Error at ") + file + ":" + std::to_string(line) + " / " + func + ": " +
                             cudaGetErrorString(result));
}

#define CUDA_CHECK(val) check_cuda_error((val), #val, __FILE__, __LINE__)

#ifndef NDEBUG
#include <iomanip>
#include <iostream>
// Prints the first n values of a device array after the stream (or the whole
// device, for stream 0) has finished.
template <typename T>
void debug_dump_device_array(const T* d_ptr, std::size_t n, const char* name, cudaStream_t stream = 0)
{
    if (n == 0) return;
    CUDA_CHECK(stream == 0 ? cudaDeviceSynchronize() : cudaStreamSynchronize(stream));
    std::vector<T> h(n);
    CUDA_CHECK(cudaMemcpy(h.data(), d_ptr, n * sizeof(T), cudaMemcpyDeviceToHost));
    std::cout << "[DEBUG] " << name << " (first " << n << " values):\n";
    for (std::size_t i = 0; i < n; ++i) std::cout << "  [" << i << "] = " << h[i] << "\n";
}

template <>
inline void debug_dump_device_array<double3>(const double3* d_ptr, std::size_t n, const char* name,
                                            cudaStream_t stream)
{
    if (n == 0) return;
    CUDA_CHECK(stream == 0 ? cudaDeviceSynchronize() : cudaStreamSynchronize(stream));
    std::vector<double3> h(n);
    cudaMemcpyAsync(h.data(), d_ptr, n * sizeof(double3), cudaMemcpyDeviceToHost, stream);
    cudaStreamSynchronize(stream);
    std::cout << name << ":\n";
    std::ios saved(nullptr);
    saved.copyfmt(std::cout);
    std::cout << std::scientific << std::setprecision(3);
    for (std::size_t i = 0; i < n; ++i)
        std::cout << "  [" << i << "] = (" << h[i].x << ", " << h[i].y << ", " << h[i].z << ")\n";
    std::cout.copyfmt(saved);
}
#endif

template <typename T>
struct HostDeviceArray1D
{
private:
    std::vector<T> h_data;
    size_t d_size{0};

public:
    T* d_ptr{nullptr};

private:
    // for the destructor and moves: no error checks, the runtime may be
    // shutting down
    void dropDevice() noexcept
    {
        if (d_ptr) (void)cudaFree(d_ptr);
        d_ptr = nullptr;
        d_size = 0;
    }

public:
    HostDeviceArray1D() = default;
    ~HostDeviceArray1D() { dropDevice(); }
    HostDeviceArray1D(const HostDeviceArray1D&) = delete;
    HostDeviceArray1D& operator=(const HostDeviceArray1D&) = delete;
    HostDeviceArray1D(HostDeviceArray1D&& other) noexcept { *this = std::move(other); }
    HostDeviceArray1D& operator=(HostDeviceArray1D&& other) noexcept
    {
        if (this != &other) {
            dropDevice();
            h_data = std::move(other.h_data);
            d_ptr = std::exchange(other.d_ptr, nullptr);
            d_size = std::exchange(other.d_size, 0);
        }
        return *this;
    }

    size_t hostSize() const { return h_data.size(); }
    size_t deviceSize() const { return d_size; }
    double deviceMemoryGB() const { return (double)d_size * sizeof(T) / (1024.0 * 1024.0 * 1024.0); }

    void releaseDevice(cudaStream_t stream)
    {
        if (d_ptr) cudaFreeAsync(d_ptr, stream);
        d_ptr = nullptr;
        d_size = 0;
    }

    void releaseDeviceSync()
    {
        if (d_ptr) cudaFree(d_ptr);
        d_ptr = nullptr;
        d_size = 0;
    }

    // n elements on the device (any previous allocation released first),
    // zeroed unless zeroFill is false
    void allocateDevice(size_t n, cudaStream_t stream, bool zeroFill = true)
    {
        if (d_ptr) releaseDevice(stream);
        d_size = n;
        if (n == 0) return;
        cudaMallocAsync((void**)&d_ptr, n * sizeof(T), stream);
        if (zeroFill) cudaMemsetAsync(d_ptr, 0, n * sizeof(T), stream);
    }

    void pushHost(const T& value) { h_data.push_back(value); }
    // inserts before index; at or past the end it appends
    void insertHost(size_t index, const T& value)
    {
        if (index >= h_data.size()) h_data.push_back(value);
        else h_data.insert(h_data.begin() + (std::ptrdiff_t)index, value);
    }
    // no-op past the end
    void eraseHost(size_t index)
    {
        if (index < h_data.size()) h_data.erase(h_data.begin() + (std::ptrdiff_t)index);
    }
    void clearHost() { h_data.clear(); }
    void reserveHost(size_t n) { h_data.reserve(n); }
    void resizeHost(size_t n) { h_data.resize(n); }
    const std::vector<T>& hostRef() const { return h_data; }
    void setHost(const std::vector<T>& values) { h_data = values; }

    // the host vector to the device, reallocating (not zeroed) when the
    // sizes differ
    void copyHostToDevice(cudaStream_t stream)
    {
        const size_t n = h_data.size();
        if (n != d_size || d_ptr == nullptr) allocateDevice(n, stream, false);
        if (n > 0) cudaMemcpyAsync(d_ptr, h_data.data(), n * sizeof(T), cudaMemcpyHostToDevice, stream);
    }

    // the device array to the host vector (resized to the device size);
    // complete once the stream reaches it
    void copyDeviceToHost(cudaStream_t stream)
    {
        if (d_size == 0 || d_ptr == nullptr) return;
        if (h_data.size() != d_size) h_data.resize(d_size);
        cudaMemcpyAsync(h_data.data(), d_ptr, d_size * sizeof(T), cudaMemcpyDeviceToHost, stream);
    }

    // a synchronous device-to-host copy, returned by value
    std::vector<T> getHostCopy()
    {
        if (d_size > 0 && d_ptr) {
            if (h_data.size() != d_size) h_data.resize(d_size);
            cudaMemcpy(h_data.data(), d_ptr, d_size * sizeof(T), cudaMemcpyDeviceToHost);
        }
        return h_data;
    }
};
