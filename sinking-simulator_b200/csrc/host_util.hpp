// host_util.hpp -- host helpers shared by the C-ABI implementations.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <string>
#include <thread>
#include <vector>

namespace fs {

// Thread-local text of the last failure raised before a handle existed.
void set_last_error(const std::string& what);
const char* last_error();

// FEMSTEP_OK when a CUDA device is usable, FEMSTEP_SKIP (with the reason recorded)
// when there is none -- the reference's "degrade, not abort" (fem_gpu.hpp:21-22).
int device_status();

// Device memory from the current device's stream-ordered pool (cudaMallocAsync on the
// legacy stream, then a wait for it, so the memory is ready for any stream).  Memory a
// handle frees stays with the process for the next handle, up to kRetainedDeviceBytes
// kept across synchronisations, instead of going back to the driver: a pool or solver
// created after another one was destroyed maps no new memory, and a destroy never waits
// in the driver's unmapping.
constexpr size_t kRetainedDeviceBytes = size_t(16) << 30;
cudaError_t device_alloc(void** p, size_t bytes);
void device_free(void* p);

// Every device allocation a handle makes, freed together.  Upload failures are sticky
// so a constructor can do all its uploads and check once.
class DeviceArena {
public:
    template <typename T>
    T* alloc(size_t count) {
        if (status_ != cudaSuccess) return nullptr;
        void* p = nullptr;
        const size_t bytes = count ? count * sizeof(T) : sizeof(T);
        status_ = device_alloc(&p, bytes);
        if (status_ != cudaSuccess) return nullptr;
        ptrs_.push_back(p);
        bytes_ += bytes;
        return static_cast<T*>(p);
    }
    template <typename T>
    T* upload(const T* host, size_t count) {
        T* d = alloc<T>(count);
        if (d && count) status_ = cudaMemcpy(d, host, count * sizeof(T), cudaMemcpyHostToDevice);
        return d;
    }
    template <typename T>
    T* zeros(size_t count) {
        T* d = alloc<T>(count);
        if (d) status_ = cudaMemset(d, 0, (count ? count : 1) * sizeof(T));
        return d;
    }
    bool ok() const { return status_ == cudaSuccess; }
    cudaError_t status() const { return status_; }
    size_t bytes() const { return bytes_; }
    void release() {
        for (void* p : ptrs_) device_free(p);
        ptrs_.clear();
        bytes_ = 0;
    }

private:
    std::vector<void*> ptrs_;
    size_t bytes_ = 0;
    cudaError_t status_ = cudaSuccess;
};

// computeRestState (engine/sim/fem.cpp:119-158) in double from float positions:
// Dm^-1 (column-major, singular guard), |det|/6, lumped rho V / 4 per corner.  The
// FP64 tet step's rest state, bit-identical to the FP64 oracle's.
void tet_rest_state64(size_t nodes, size_t tets, const float* position, const uint32_t* index, double density,
                      std::vector<double>& inv, std::vector<double>& vol, std::vector<double>& mass);

// f(begin, end) over [0, n) split into contiguous chunks, one per host core (inline
// when n is small).  For loops whose iterations are independent.
template <class F>
void parallel_chunks(size_t n, F f, size_t min_chunk = size_t(1) << 16) {
    const size_t cores = std::max(1u, std::thread::hardware_concurrency());
    const size_t parts = std::min(cores, std::max<size_t>(1, n / min_chunk));
    if (parts <= 1) {
        f(size_t(0), n);
        return;
    }
    std::vector<std::thread> pool;
    for (size_t k = 0; k < parts; ++k) {
        const size_t b = n * k / parts, e = n * (k + 1) / parts;
        pool.emplace_back([=, &f]() { f(b, e); });
    }
    for (auto& t : pool) t.join();
}

// Node -> incident corner CSR by counting sort, the construction of
// engine/sim/fem.cpp:147-157 and engine/sim/zone.cpp:739-754.
inline void build_csr(size_t nodes, size_t elements, int corners, const uint32_t* index,
                      std::vector<uint32_t>& offset, std::vector<uint32_t>& entry) {
    offset.assign(nodes + 1, 0u);
    for (size_t e = 0; e < elements; ++e)
        for (int c = 0; c < corners; ++c) ++offset[index[e * corners + c] + 1];
    for (size_t n = 0; n < nodes; ++n) offset[n + 1] += offset[n];
    entry.assign(elements * corners, 0u);
    std::vector<uint32_t> cursor(offset.begin(), offset.end() - 1);
    for (size_t e = 0; e < elements; ++e)
        for (int c = 0; c < corners; ++c)
            entry[cursor[index[e * corners + c]]++] = (uint32_t)e * (uint32_t)corners + (uint32_t)c;
}

}  // namespace fs
