// tet_fast.cu -- the single-mesh FP32 J2 tet step, plain and Kahan-compensated.
//
// The element and node updates are in tet_f32.cuh (shared with the batched pool);
// this file maps them one thread per tet / per node and keeps the energy account as
// FP64 per-block partials, which the host reduces on the device in fixed order.
#include "common.cuh"
#include "tet.hpp"
#include "tet_f32.cuh"

namespace fs {
namespace {

// The FP32 modes keep disp / disp_c as float4 per node and slots as float4 per corner.
__device__ __forceinline__ TetElementRefs refs(const TetDevice<float>& d) {
    return TetElementRefs{d.index,
                          d.slot,
                          d.rest_inv,
                          d.rest_vol,
                          d.plastic,
                          d.plastic_c,
                          reinterpret_cast<const float4*>(d.disp),
                          reinterpret_cast<const float4*>(d.disp_c),
                          reinterpret_cast<float4*>(d.slots),
                          d.tets};
}

// 1024 / kBlock blocks per SM: 64 registers, 32 resident warps per SM
template <bool KAHAN>
__global__ void __launch_bounds__(kBlock, 1024 / kBlock) f32_forces(TetDevice<float> d, J2f m, int wave) {
    __shared__ double scratch[64];
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    {
        // the rows of the block one wave later, into L2
        const long long nb = (long long)(blockIdx.x + wave) * blockDim.x;
        const long long ne = nb + blockDim.x < d.tets ? nb + blockDim.x : d.tets;
        prefetch_tet_rows(refs(d), nb, ne);
    }
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const long long s = d.counter[0];
        d.counter[1] = s;
        d.counter[0] = s + 1;
    }
    double diss = 0.0, energy = 0.0;
    if (t < d.tets) {
        tet_element_f32<KAHAN>(refs(d), t, m, diss, energy);
    }
    block_sum2(diss, energy, scratch);  // valid in thread 0
    if (threadIdx.x == 0) {
        d.e_diss[blockIdx.x] += diss;
        d.e_strain[blockIdx.x] = energy;
    }
}

template <bool KAHAN>
__global__ void __launch_bounds__(kBlock) f32_nodes(TetDevice<float> d, float dt, float gravity, float damping,
                                                    int ramp) {
    __shared__ double scratch[32];
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double work = 0.0, kin = 0.0, gwork = 0.0;
    if (n < d.nodes) {
        const TetNodeRefs r{d.offset,   reinterpret_cast<const float4*>(d.slots), d.fixed,
                            d.mass,     d.inv_mass,
                            d.ext,      d.velocity,
                            reinterpret_cast<float4*>(d.disp), reinterpret_cast<float4*>(d.disp_c)};
        const float lf = (float)ramp_factor(d.counter[1], ramp);
        tet_node_f32<KAHAN>(r, n, lf, dt, gravity, damping, work, kin, gwork);
    }
    const double bw = block_sum(work, scratch);
    const double bk = block_sum(kin, scratch);
    const double bg = block_sum(gwork, scratch);
    if (threadIdx.x == 0) {
        d.n_work[blockIdx.x] += bw;
        d.n_kin[blockIdx.x] = bk;
        d.n_grav[blockIdx.x] += bg;
    }
}

}  // namespace

void launch_f32_step(const TetDevice<float>& d, const TetParams& p, bool compensated, cudaStream_t stream,
                     int parts) {
    const int eb = blocks_for(d.tets, kBlock), nb = blocks_for(d.nodes, kBlock);
    const J2f m = make_j2f(p.mu, p.bulk, p.yield, p.hardening);
    const int wave = sm_count() * (1024 / kBlock);
    if (compensated) {
        if (parts & kElementPart) f32_forces<true><<<eb, kBlock, 0, stream>>>(d, m, wave);
        if (parts & kNodePart)
            f32_nodes<true><<<nb, kBlock, 0, stream>>>(d, (float)p.dt, (float)p.gravity, (float)p.damping, p.ramp);
    } else {
        if (parts & kElementPart) f32_forces<false><<<eb, kBlock, 0, stream>>>(d, m, wave);
        if (parts & kNodePart)
            f32_nodes<false><<<nb, kBlock, 0, stream>>>(d, (float)p.dt, (float)p.gravity, (float)p.damping, p.ramp);
    }
}

}  // namespace fs
