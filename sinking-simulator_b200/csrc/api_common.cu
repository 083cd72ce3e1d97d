// api_common.cu -- error text and device discovery shared by every entry point.
#include <cuda_runtime.h>

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
