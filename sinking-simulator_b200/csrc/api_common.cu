// api_common.cu -- error text and device discovery shared by every entry point.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>

#include "../../include/femstep.h"
#include "host_util.hpp"

namespace fs {

namespace {
thread_local std::string g_last_error;
}

void set_last_error(const std::string& what) { g_last_error = what; }
const char* last_error() { return g_last_error.c_str(); }

cudaError_t device_alloc(void** p, size_t bytes) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    // once per device: keep freed memory up to the retained size
    static bool configured[64] = {};
    if (dev >= 0 && dev < 64 && !configured[dev]) {
        cudaMemPool_t pool = nullptr;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t keep = kRetainedDeviceBytes;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        configured[dev] = true;
    }
    e = cudaMallocAsync(p, bytes, cudaStreamLegacy);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(cudaStreamLegacy);
}

void device_free(void* p) {
    if (p) cudaFreeAsync(p, cudaStreamLegacy);
}

int device_status() {
    int count = 0;
    const cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        set_last_error(std::string("no CUDA device (") + (e != cudaSuccess ? cudaGetErrorString(e) : "count 0") + ")");
        cudaGetLastError();
        return FEMSTEP_SKIP;
    }
    return FEMSTEP_OK;
}

void tet_rest_state64(size_t nodes, size_t tets, const float* position, const uint32_t* index, double density,
                      std::vector<double>& inv, std::vector<double>& vol, std::vector<double>& mass) {
    inv.assign(tets * 9, 0.0);
    vol.assign(tets, 0.0);
    mass.assign(nodes, 0.0);
    for (size_t t = 0; t < tets; ++t) {
        const uint32_t* idx = &index[t * 4];
        double a[9];  // column-major
        for (int c = 0; c < 3; ++c)
            for (int r = 0; r < 3; ++r)
                a[c * 3 + r] = (double)position[(size_t)idx[c + 1] * 3 + r] - (double)position[(size_t)idx[0] * 3 + r];
#define A(r, c) a[(c) * 3 + (r)]
        const double det = A(0, 0) * (A(1, 1) * A(2, 2) - A(1, 2) * A(2, 1)) -
                           A(0, 1) * (A(1, 0) * A(2, 2) - A(1, 2) * A(2, 0)) +
                           A(0, 2) * (A(1, 0) * A(2, 1) - A(1, 1) * A(2, 0));
        const double volume = det / 6.0;
        vol[t] = std::fabs(volume);
        const double id = std::fabs(det) > 1e-300 ? 1.0 / det : 0.0;
        double* r = &inv[t * 9];
#define R(rr, cc) r[(cc) * 3 + (rr)]
        R(0, 0) = (A(1, 1) * A(2, 2) - A(1, 2) * A(2, 1)) * id;
        R(0, 1) = (A(0, 2) * A(2, 1) - A(0, 1) * A(2, 2)) * id;
        R(0, 2) = (A(0, 1) * A(1, 2) - A(0, 2) * A(1, 1)) * id;
        R(1, 0) = (A(1, 2) * A(2, 0) - A(1, 0) * A(2, 2)) * id;
        R(1, 1) = (A(0, 0) * A(2, 2) - A(0, 2) * A(2, 0)) * id;
        R(1, 2) = (A(0, 2) * A(1, 0) - A(0, 0) * A(1, 2)) * id;
        R(2, 0) = (A(1, 0) * A(2, 1) - A(1, 1) * A(2, 0)) * id;
        R(2, 1) = (A(0, 1) * A(2, 0) - A(0, 0) * A(2, 1)) * id;
        R(2, 2) = (A(0, 0) * A(1, 1) - A(0, 1) * A(1, 0)) * id;
#undef R
#undef A
        const double quarter = density * vol[t] * 0.25;
        for (int c = 0; c < 4; ++c) mass[idx[c]] += quarter;
    }
}

}  // namespace fs

extern "C" {

const char* femstep_last_error(void) { return fs::last_error(); }

int femstep_set_device(int device) {
    const int st = fs::device_status();
    if (st != FEMSTEP_OK) return st;
    const cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        fs::set_last_error(std::string("cudaSetDevice: ") + cudaGetErrorString(e));
        return FEMSTEP_EINVAL;
    }
    return FEMSTEP_OK;
}

int femstep_device_name(char* buffer, size_t length) {
    const int st = fs::device_status();
    if (st != FEMSTEP_OK) return st;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return FEMSTEP_ECUDA;
    if (buffer && length) {
        std::strncpy(buffer, prop.name, length - 1);
        buffer[length - 1] = '\0';
    }
    return FEMSTEP_OK;
}

}  // extern "C"
