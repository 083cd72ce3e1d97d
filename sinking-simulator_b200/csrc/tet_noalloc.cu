// tet_noalloc.cu -- the REF32 tet step for callers that cannot allocate device memory.
//
// Some callers own every byte of device memory themselves: a host engine with its own
// arena allocator, a plugin loaded into a process whose memory budget is fixed, code
// that runs where cudaMalloc is not allowed or not wanted (a capped memory pool, a
// real-time loop that must never block on the allocator).  Such a caller already has
// the mesh in device memory and wants the step applied to it, but femstep_tet_create
// allocates: the device copy of the mesh and the per-tet force scratch.
//
// femstep_tet_step_noalloc takes the caller's device arrays in the reference's own
// TetMesh layout (engine/sim/fem.hpp:38-68) and keeps its only scratch -- the twelve
// corner forces of every tet, the reference's TetMesh::tetForce -- in a file-scope
// __device__ array of a fixed size, g_force_scratch below.  It calls no cudaMalloc,
// no cudaFree and no allocating library routine.  The arithmetic is fem::tetForces and
// fem::stepCpu's (engine/sim/fem.cpp:73-117, 187-215) in the same order, compiled
// without FMA contraction, so the result is bit-identical to FEMSTEP_TET_REF32 and to
// the reference CPU step.
//
// The array costs kNoAllocMaxTets * 48 bytes (3 MiB) on every GPU that loads the
// library, for as long as the process lives.  Every call on a device shares it, so
// two calls whose kernels overlap on that GPU (different streams, different threads)
// race on it; calls on one stream are ordered and safe.  It keeps the last call's
// contents; nothing needs clearing because each step writes every tet's twelve slots
// before the node pass reads them.
//
// The array's device address belongs to one CUDA context.  The first call in a
// context looks it up (cudaGetSymbolAddress, with that context's device current) and
// keeps it keyed on the context's process-unique id, so a new context on the same
// device -- after cudaDeviceReset, or a caller's own driver-API context -- gets its
// own lookup.  Make that first call outside any stream capture.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/femstep.h"
#include "common.cuh"
#include "host_util.hpp"

// The whole of the entry point's scratch: twelve corner forces per tet for up to
// 65,536 tets (3 MiB), resident on every GPU that loads the library.
static __device__ __align__(256) float g_force_scratch[65536 * 12];

namespace fs {
namespace {

constexpr long long kNoAllocMaxTets = 65536;
constexpr int kMaxDevices = 64;

// Device address of g_force_scratch per device, looked up with that device current
// and kept with the id of the context it belongs to.  In host code the symbol is only
// a host-side stand-in and must never be handed to a kernel.
struct ScratchAddress {
    unsigned long long context = 0;  // cuCtxGetId of the context the address is valid in
    float* ptr = nullptr;
};
ScratchAddress g_scratch[kMaxDevices];
std::mutex g_scratch_mutex;

__device__ __forceinline__ M3<float> polar4(const M3<float>& f) {
    M3<float> r = f;
#pragma unroll 1
    for (int i = 0; i < 4; ++i) {
        const M3<float> rit = transpose(inverse(r, 1e-30f));
#pragma unroll
        for (int k = 0; k < 9; ++k) r.m[k] = 0.5f * (r.m[k] + rit.m[k]);
    }
    return r;
}

// fem::tetForces (fem.cpp:73-117), written to the tet-major scratch like TetMesh::tetForce.
__global__ void __launch_bounds__(kBlock) noalloc_forces(femstep_tet_device_mesh m, float* scratch, float lambda,
                                                          float mu) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)m.tets) return;
    const uint32_t* idx = m.index + t * 4;
    const float* p = m.position;
    M3<float> ds, dm_inv;
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int a = 0; a < 3; ++a) ds(a, c) = p[(size_t)idx[c + 1] * 3 + a] - p[(size_t)idx[0] * 3 + a];
#pragma unroll
    for (int k = 0; k < 9; ++k) dm_inv.m[k] = m.rest_inv[t * 9 + k];
    const M3<float> f = mul(ds, dm_inv);
    const M3<float> r = polar4(f);
    const M3<float> s = mul(transpose(r), f);
    M3<float> strain;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) strain(i, j) = 0.5f * (s(i, j) + s(j, i));
#pragma unroll
    for (int i = 0; i < 3; ++i) strain(i, i) -= 1.0f;
    const float trace = strain(0, 0) + strain(1, 1) + strain(2, 2);
    M3<float> stress;
#pragma unroll
    for (int k = 0; k < 9; ++k) stress.m[k] = 2.0f * mu * strain.m[k];
#pragma unroll
    for (int i = 0; i < 3; ++i) stress(i, i) += lambda * trace;
    const M3<float> h = mul(mul(r, stress), transpose(dm_inv));
    const float scale = -m.rest_volume[t];
    float* out = scratch + t * 12;
    float f0[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float v = scale * h(a, c);
            out[(c + 1) * 3 + a] = v;
            f0[a] -= v;
        }
#pragma unroll
    for (int a = 0; a < 3; ++a) out[a] = f0[a];
}

// fem::stepCpu's node loop (fem.cpp:196-214) over the reference's own CSR.
__global__ void __launch_bounds__(kBlock) noalloc_nodes(femstep_tet_device_mesh m, const float* scratch, float dt,
                                                         float gravity, float damping) {
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= (long long)m.nodes) return;
    float* vel = m.velocity + n * 3;
    if (m.fixed && m.fixed[n]) {
        vel[0] = 0.0f;
        vel[1] = 0.0f;
        vel[2] = 0.0f;
        return;
    }
    const float mass = m.mass[n];
    float force[3] = {0.0f, 0.0f, -gravity * mass};
    for (uint32_t e = m.adjacency_offset[n]; e < m.adjacency_offset[n + 1]; ++e) {
        const uint32_t entry = m.adjacency_entry[e];
        const float* f = scratch + (size_t)(entry >> 2) * 12 + (entry & 3u) * 3;
        force[0] += f[0];
        force[1] += f[1];
        force[2] += f[2];
    }
    const float inv_mass = 1.0f / mass;
    float* pos = m.position + n * 3;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float v = vel[k] + force[k] * inv_mass * dt;
        v *= damping;
        vel[k] = v;
        pos[k] += v * dt;
    }
}

// The id of the current context, through the driver's entry points as the runtime
// hands them out (no link to the driver library).  0 when there is none.
unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(fn);
        fn = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(fn);
    });
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

int scratch_for_current_device(float** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_last_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
        return FEMSTEP_ECUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        set_last_error("device ordinal beyond the no-allocation entry point's table");
        return FEMSTEP_EINVAL;
    }
    // Before the runtime's first use of the device there is no current context (id 0):
    // the lookup then brings it up, and the address is kept under its id.  If the
    // context cannot be named at all, the address is looked up on every call.
    const unsigned long long ctx = current_context_id();
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    ScratchAddress& slot = g_scratch[dev];
    if (!slot.ptr || ctx == 0 || slot.context != ctx) {
        float* p = nullptr;
        e = cudaGetSymbolAddress((void**)&p, ::g_force_scratch);
        if (e != cudaSuccess || !p) {
            set_last_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            return FEMSTEP_ECUDA;
        }
        slot.ptr = p;
        slot.context = ctx ? ctx : current_context_id();
    }
    *out = slot.ptr;
    return FEMSTEP_OK;
}

}  // namespace
}  // namespace fs

extern "C" {

int femstep_tet_step_noalloc(const femstep_tet_device_mesh* mesh, int substeps, const femstep_tet_params* params,
                             void* stream) {
    if (!mesh || !params) {
        fs::set_last_error("null mesh or params");
        return FEMSTEP_EINVAL;
    }
    const femstep_tet_device_mesh& m = *mesh;
    if (m.tets == 0 || m.nodes == 0 || !m.position || !m.velocity || !m.mass || !m.index || !m.rest_inv ||
        !m.rest_volume || !m.adjacency_offset || !m.adjacency_entry) {
        fs::set_last_error("every array except `fixed` is required");
        return FEMSTEP_EINVAL;
    }
    if (m.tets > (size_t)fs::kNoAllocMaxTets) {
        fs::set_last_error("femstep_tet_step_noalloc: " + std::to_string(m.tets) + " tets exceed its fixed scratch of " +
                           std::to_string(fs::kNoAllocMaxTets) + " tets; use femstep_tet_create");
        return FEMSTEP_EINVAL;
    }
    if (substeps < 0 || !(params->dt > 0.0)) {
        fs::set_last_error("negative step count or non-positive dt");
        return FEMSTEP_EINVAL;
    }
    if (params->yield_strength > 0.0 || params->hardening_modulus != 0.0 || params->ramp_steps != 0) {
        fs::set_last_error("femstep_tet_step_noalloc is the elastic REF32 step: yield_strength, hardening_modulus "
                           "and ramp_steps must be 0");
        return FEMSTEP_EINVAL;
    }
    const int dev = fs::device_status();
    if (dev != FEMSTEP_OK) return dev;
    // an error left by an earlier call on this thread is reported as such, not as this
    // call's launch failure
    const cudaError_t pending = cudaGetLastError();
    if (pending != cudaSuccess) {
        fs::set_last_error(std::string("a CUDA error from before this call was pending: ") +
                           cudaGetErrorString(pending));
        return FEMSTEP_ECUDA;
    }
    float* scratch = nullptr;
    const int rc = fs::scratch_for_current_device(&scratch);
    if (rc) return rc;
    // fem::Material::lameLambda / lameMu in float (fem.hpp:29-33)
    const float E = (float)params->youngs_modulus, nu = (float)params->poisson_ratio;
    const float lambda = E * nu / ((1.0f + nu) * (1.0f - 2.0f * nu));
    const float mu = E / (2.0f * (1.0f + nu));
    const cudaStream_t s = (cudaStream_t)stream;
    const int eb = fs::blocks_for((long long)m.tets, fs::kBlock), nb = fs::blocks_for((long long)m.nodes, fs::kBlock);
    for (int i = 0; i < substeps; ++i) {
        fs::noalloc_forces<<<eb, fs::kBlock, 0, s>>>(m, scratch, lambda, mu);
        fs::noalloc_nodes<<<nb, fs::kBlock, 0, s>>>(m, scratch, (float)params->dt, (float)params->gravity,
                                                    (float)params->damping);
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fs::set_last_error(std::string("femstep_tet_step_noalloc launch: ") + cudaGetErrorString(e));
        return FEMSTEP_ECUDA;
    }
    return FEMSTEP_OK;
}

}  // extern "C"
