// common.cuh -- shared device helpers for the femstep kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fs {

constexpr int kBlock = 256;  // threads per block for the element and node kernels

inline int blocks_for(long long n, int block) { return (int)((n + block - 1) / block); }

// SMs of the current device.
inline int sm_count() {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms > 0 ? sms : 1;
}

// Deterministic block sum in double: shuffle tree inside each warp, then warp 0 adds
// the per-warp partials in warp order.  The association order depends only on the
// block size, never on scheduling, so the same launch always produces the same bits.
__device__ __forceinline__ double block_sum(double v, double* scratch /* >= 32 */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    double total = 0.0;
    if (threadIdx.x == 0) {
        const int warps = (blockDim.x + 31) >> 5;
        for (int w = 0; w < warps; ++w) total += scratch[w];
    }
    __syncthreads();
    return total;  // valid in thread 0 only
}

// Two deterministic block sums in one pass (one pair of barriers): the same order as
// block_sum for each.  scratch >= 64 doubles.
// The warp part of block_sum2: each of a and b summed over the warp into lane 0.
__device__ __forceinline__ void warp_sum2(double& a, double& b) {
    // a warp whose `a` values are all zero (no tet yielded) has the sum zero already
    if (__any_sync(0xffffffffu, a != 0.0)) {
        for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    }
    for (int o = 16; o > 0; o >>= 1) b += __shfl_down_sync(0xffffffffu, b, o);
}

__device__ __forceinline__ void block_sum2(double& a, double& b, double* scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    warp_sum2(a, b);
    if (lane == 0) {
        scratch[warp] = a;
        scratch[32 + warp] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int warps = (blockDim.x + 31) >> 5;
        double ta = 0.0, tb = 0.0;
        for (int w = 0; w < warps; ++w) {
            ta += scratch[w];
            tb += scratch[32 + w];
        }
        a = ta;
        b = tb;
    }
    __syncthreads();
}

// Column-major 3x3, the layout engine/sim/fem.cpp uses for its M3.
template <typename T>
struct M3 {
    T m[9];
    __device__ __forceinline__ T& operator()(int r, int c) { return m[c * 3 + r]; }
    __device__ __forceinline__ T operator()(int r, int c) const { return m[c * 3 + r]; }
};

template <typename T>
__device__ __forceinline__ M3<T> mul(const M3<T>& a, const M3<T>& b) {
    M3<T> r;
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            T s = T(0);
#pragma unroll
            for (int k = 0; k < 3; ++k) s += a(i, k) * b(k, c);
            r(i, c) = s;
        }
    return r;
}

template <typename T>
__device__ __forceinline__ M3<T> transpose(const M3<T>& a) {
    M3<T> r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r(i, j) = a(j, i);
    return r;
}

template <typename T>
__device__ __forceinline__ T det3(const M3<T>& a) {
    return a(0, 0) * (a(1, 1) * a(2, 2) - a(1, 2) * a(2, 1)) -
           a(0, 1) * (a(1, 0) * a(2, 2) - a(1, 2) * a(2, 0)) +
           a(0, 2) * (a(1, 0) * a(2, 1) - a(1, 1) * a(2, 0));
}

// Adjugate over the determinant, with the reference's singular guard
// (engine/sim/fem.cpp:42-56): a determinant at or below `tiny` gives the zero matrix.
template <typename T>
__device__ __forceinline__ M3<T> inverse(const M3<T>& a, T tiny) {
    const T det = det3(a);
    const T id = fabs(det) > tiny ? T(1) / det : T(0);
    M3<T> r;
    r(0, 0) = (a(1, 1) * a(2, 2) - a(1, 2) * a(2, 1)) * id;
    r(0, 1) = (a(0, 2) * a(2, 1) - a(0, 1) * a(2, 2)) * id;
    r(0, 2) = (a(0, 1) * a(1, 2) - a(0, 2) * a(1, 1)) * id;
    r(1, 0) = (a(1, 2) * a(2, 0) - a(1, 0) * a(2, 2)) * id;
    r(1, 1) = (a(0, 0) * a(2, 2) - a(0, 2) * a(2, 0)) * id;
    r(1, 2) = (a(0, 2) * a(1, 0) - a(0, 0) * a(1, 2)) * id;
    r(2, 0) = (a(1, 0) * a(2, 1) - a(1, 1) * a(2, 0)) * id;
    r(2, 1) = (a(0, 1) * a(2, 0) - a(0, 0) * a(2, 1)) * id;
    r(2, 2) = (a(0, 0) * a(1, 1) - a(0, 1) * a(1, 0)) * id;
    return r;
}

// Load factor of a linear ramp over `ramp` steps, evaluated for the step that is
// about to be taken: min((step + 1) / ramp, 1).
__device__ __forceinline__ double ramp_factor(long long step, int ramp) {
    if (ramp <= 0) return 1.0;
    const double f = (double)(step + 1) / (double)ramp;
    return f < 1.0 ? f : 1.0;
}

}  // namespace fs
