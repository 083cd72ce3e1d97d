// tet.hpp -- device-side layout of a tet mesh and the kernel launchers.
//
// Device layout (built by api.cu from the reference's host TetMesh, fem.hpp:38-68):
//
//   per tet, structure-of-arrays so a warp's loads are contiguous:
//     index      uint4   [T]      the four node ids
//     slot       uint4   [T]      where each corner's force goes in the node-major
//                                 slot array: slot[t].c = position of entry t*4+c in
//                                 the CSR (the inverse permutation of adjacencyEntry)
//     rest_inv   Real    [9][T]   Dm^-1, column-major per tet
//     rest_vol   Real    [T]
//     plastic    Real    [7][T]   plastic strain (6, engineering shears), eq. plastic strain
//     plastic_c  float   [7][T]   Kahan compensation (FP32-compensated mode only)
//   per node:
//     position / rest   Real  [3N]   (reference AoS x,y,z)
//     disp, disp_c      float [4N]   displacement and its compensation (FP32 modes),
//                                    one (x, y, z, 0) float4 per node
//     velocity          Real  [3N]
//     mass, inv_mass    Real  [N]
//     fixed             uint8 [N]
//     offset            uint32[N+1]  CSR offsets (adjacencyOffset)
//     ext               Real  [3N]   full-load external force (optional)
//   per CSR entry (node-major, the reference's gather order):
//     slots             Real  [3 * 4T] (REF32, FP64); float4 [4T] (FP32 J2 modes)
//
// The element kernel writes each corner force straight to its node-major slot, so the
// node kernel reads its incident forces as one contiguous run and sums them in exactly
// the reference's CSR order.  No float atomics anywhere; the result does not depend on
// scheduling.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fs {

template <typename Real>
struct TetDevice {
    long long nodes = 0, tets = 0;
    // elements
    const uint4* index = nullptr;
    const uint4* slot = nullptr;
    const Real* rest_inv = nullptr;
    const Real* rest_vol = nullptr;
    Real* plastic = nullptr;
    float* plastic_c = nullptr;
    // nodes
    Real* position = nullptr;   // REF32 / F64: current positions
    const float* rest = nullptr;  // FP32 J2 modes: rest positions
    float* disp = nullptr;        // FP32 J2 modes
    float* disp_c = nullptr;      // FP32 compensated
    Real* velocity = nullptr;
    const Real* mass = nullptr;
    const Real* inv_mass = nullptr;
    const uint8_t* fixed = nullptr;
    const uint32_t* offset = nullptr;
    const Real* ext = nullptr;
    Real* slots = nullptr;
    // step bookkeeping: counter[0] = steps taken, counter[1] = step the node kernel of
    // the current step uses (written by the element kernel's first thread)
    long long* counter = nullptr;
    // FP64 energy partials, one entry per block, fixed block->data mapping:
    //   e_diss (+=), e_strain (=) per element block;
    //   n_work (+=), n_kin (=), n_grav (+=) per node block
    double* e_diss = nullptr;
    double* e_strain = nullptr;
    double* n_work = nullptr;
    double* n_kin = nullptr;
    double* n_grav = nullptr;
};

struct TetParams {
    double lambda, mu, bulk;      // Lame constants and bulk modulus
    double yield, hardening;      // J2 linear isotropic hardening
    double dt, gravity, damping;
    int ramp;
};

// Launchers.  `stream` is the caller's stream; every launch is asynchronous.
// `parts`: kElementPart | kNodePart (a whole step), or one of them alone (profiling).
constexpr int kElementPart = 1, kNodePart = 2, kWholeStep = 3;
void launch_ref32_step(const TetDevice<float>& d, const TetParams& p, cudaStream_t stream,
                       int parts = kWholeStep);
void launch_f64_step(const TetDevice<double>& d, const TetParams& p, cudaStream_t stream,
                     int parts = kWholeStep);
void launch_f32_step(const TetDevice<float>& d, const TetParams& p, bool compensated,
                     cudaStream_t stream, int parts = kWholeStep);
// FP64 element eigenvalue bound: omega^2 per tet, reduced to the maximum on device.
void launch_tet_omega2(long long tets, const double* rest_inv, double E, double nu, double rho,
                       double* per_block_max, int blocks, cudaStream_t stream);
// The same bound from an FP32 Dm^-1 (SoA with stride `stride`, `rest_inv` pointing at
// the first tet), promoted to double: the matrix the FP32 element kernels use.
void launch_tet_omega2_f32(long long tets, const float* rest_inv, long long stride, double E, double nu, double rho,
                           double* per_block_max, int blocks, cudaStream_t stream);
// The single mesh's rest state on the device, bit-identical to tet_rest_state64:
// per tet Dm^-1 (SoA, `tets` per row), volume and quarter mass; per node the lumped
// mass summed over the node's CSR run (`entry`: corner ids, ascending per node).
void launch_tet_rest64(const float* position, const uint32_t* index, long long tets, double density, double* inv,
                       double* vol, double* quarter, cudaStream_t stream);
void launch_tet_mass64(const uint32_t* offset, const uint32_t* entry, long long nodes, const double* quarter,
                       double* mass, cudaStream_t stream);
// The FP32 modes' rest state from it: Dm^-1, volume, mass and 1 / mass, rounded once.
void launch_tet_rest_f32(const double* inv, const double* vol, long long tets, const double* mass, long long nodes,
                         float* inv32, float* vol32, float* mass32, float* inv_mass32, cudaStream_t stream);
// out[i] = (double)in[i].
void launch_widen(const float* in, long long n, double* out, cudaStream_t stream);
// Fixed-order FP64 sum / max of `n` doubles into out[0] (one block).
void launch_reduce_sum(const double* in, long long n, double* out, cudaStream_t stream);
void launch_reduce_max(const double* in, long long n, double* out, cudaStream_t stream);

}  // namespace fs
