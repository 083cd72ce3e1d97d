// api_tet.cu -- host side of the tet step behind the C ABI (include/femstep.h).
//
// Replaces gpu::FemGpuSolver (engine/gpu/fem_gpu.{hpp,cpp}): the same three calls
// (initialise -> femstep_tet_create, run -> femstep_tet_run, readback ->
// femstep_tet_readback) with the same ownership (the handle owns its device copy, the
// caller keeps the host mesh) and the same error convention (a status plus text;
// no device is a skip, not an abort).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/femstep.h"
#include "common.cuh"
#include "host_util.hpp"
#include "shell.hpp"
#include "tet.hpp"

using fs::TetDevice;
using fs::TetParams;

struct femstep_tet {
    int mode = 0;
    size_t nodes = 0, tets = 0;
    cudaStream_t stream = nullptr;
    fs::DeviceArena arena;
    TetDevice<float> d32;
    TetDevice<double> d64;
    std::vector<float> rest;          // FP32 J2 modes: rest positions for readback
    std::vector<double> rest_inv64;   // J2 modes given an adjacency: Dm^-1 in double (critical dt)
    double* inv64 = nullptr;          // J2 FP32 modes built on the device: Dm^-1 in double, SoA
    int eblocks = 0, nblocks = 0;
    double* d_out = nullptr;          // 8 doubles of reduction output
    double* d_scratch = nullptr;      // per-block maxima for the critical step
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    TetParams graph_params{};
    long long launches = 0;
    std::string error;
};

namespace {

int fail(femstep_tet* s, int code, const std::string& what) {
    if (s) s->error = what;
    fs::set_last_error(what);
    return code;
}

void rest_state64(const femstep_tet_mesh& m, std::vector<double>& inv, std::vector<double>& vol,
                  std::vector<double>& mass) {
    fs::tet_rest_state64(m.nodes, m.tets, m.position, m.index, m.density, inv, vol, mass);
}

template <typename T>
std::vector<T> soa(const T* aos, size_t count, int width) {
    std::vector<T> out((size_t)width * count);
    for (size_t i = 0; i < count; ++i)
        for (int k = 0; k < width; ++k) out[(size_t)k * count + i] = aos[i * width + k];
    return out;
}

int check(femstep_tet* s, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return FEMSTEP_OK;
    return fail(s, e == cudaErrorMemoryAllocation ? FEMSTEP_ENOMEM : FEMSTEP_ECUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

TetParams make_params(const femstep_tet* s, const femstep_tet_params& p) {
    TetParams q{};
    if (s->mode == FEMSTEP_TET_REF32) {
        // fem::Material::lameLambda / lameMu (fem.hpp:29-33), in float arithmetic.
        const float E = (float)p.youngs_modulus, nu = (float)p.poisson_ratio;
        q.lambda = (double)(E * nu / ((1.0f + nu) * (1.0f - 2.0f * nu)));
        q.mu = (double)(E / (2.0f * (1.0f + nu)));
    } else {
        const double E = p.youngs_modulus, nu = p.poisson_ratio;
        q.lambda = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
        // plasticity::Material::shearModulus / bulkModulus (plasticity.hpp:226-227)
        q.mu = E / (2.0 * (1.0 + nu));
        q.bulk = E / (3.0 * (1.0 - 2.0 * nu));
    }
    q.yield = p.yield_strength;
    q.hardening = p.hardening_modulus;
    q.dt = p.dt;
    q.gravity = p.gravity;
    q.damping = p.damping;
    q.ramp = p.ramp_steps;
    return q;
}

void launch_step(femstep_tet* s, const TetParams& q, int parts = fs::kWholeStep) {
    switch (s->mode) {
        case FEMSTEP_TET_REF32: fs::launch_ref32_step(s->d32, q, s->stream, parts); break;
        case FEMSTEP_TET_J2_F32: fs::launch_f32_step(s->d32, q, false, s->stream, parts); break;
        case FEMSTEP_TET_J2_F32K: fs::launch_f32_step(s->d32, q, true, s->stream, parts); break;
        default: fs::launch_f64_step(s->d64, q, s->stream, parts); break;
    }
}

constexpr int kGraphSteps = 32;

// femstep_tet_create for the J2 modes when the caller gives no adjacency (the mesh is
// already checked): everything from the caller's node positions and node ids on the
// device.  The CSR and slot map of csr.cu (counting-sort order), and computeRestState
// (fem.cpp:119-158) in FP64 by tet_exact.cu's kernels, bit-identical to the host's
// tet_rest_state64; the FP32 modes' float copies rounded once from it.
int create_on_device(const femstep_tet_mesh& m, int mode, femstep_tet** out) {
    const int dev = fs::device_status();
    if (dev != FEMSTEP_OK) return dev;
    const size_t N = m.nodes, T = m.tets;
    femstep_tet* s = new femstep_tet();
    s->mode = mode;
    s->nodes = N;
    s->tets = T;
    s->eblocks = fs::blocks_for((long long)T, fs::kBlock);
    s->nblocks = fs::blocks_for((long long)N, fs::kBlock);
    int rc = check(s, cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "stream");
    if (rc == FEMSTEP_OK) rc = check(s, cudaEventCreate(&s->ev0), "event");
    if (rc == FEMSTEP_OK) rc = check(s, cudaEventCreate(&s->ev1), "event");
    if (rc != FEMSTEP_OK) {
        femstep_tet_destroy(s);
        return rc;
    }
    fs::DeviceArena& A = s->arena;
    std::vector<uint8_t> fixed(N, 0);
    if (m.fixed)
        for (size_t n = 0; n < N; ++n) fixed[n] = m.fixed[n] ? 1 : 0;
    const uint32_t* index = A.upload(m.index, T * 4);
    const float* pos32 = A.upload(m.position, N * 3);
    uint32_t* offset = A.alloc<uint32_t>(N + 1);
    uint32_t* slot = A.alloc<uint32_t>(T * 4);
    // the FP64 rest state: Dm^-1 (SoA) and volumes per tet, lumped masses per node
    double* inv64 = A.alloc<double>(T * 9);
    double* vol64 = A.alloc<double>(T);
    double* mass64 = A.alloc<double>(N);
    if (!A.ok()) {
        const int code = A.status() == cudaErrorMemoryAllocation ? FEMSTEP_ENOMEM : FEMSTEP_ECUDA;
        fail(s, code, std::string("device upload failed: ") + cudaGetErrorString(A.status()));
        femstep_tet_destroy(s);
        return code;
    }
    uint32_t* entry = nullptr;
    double* quarter = nullptr;
    rc = check(s, fs::device_alloc((void**)&entry, T * 4 * sizeof(uint32_t)), "alloc");
    if (!rc) rc = check(s, fs::device_alloc((void**)&quarter, T * sizeof(double)), "alloc");
    if (!rc) rc = check(s, fs::build_csr_device(index, (long long)T * 4, (long long)N, offset, slot, s->stream, entry),
                        "adjacency");
    if (!rc) {
        fs::launch_tet_rest64(pos32, index, (long long)T, m.density, inv64, vol64, quarter, s->stream);
        fs::launch_tet_mass64(offset, entry, (long long)N, quarter, mass64, s->stream);
        rc = check(s, cudaGetLastError(), "rest state");
    }

    auto common = [&](auto& d) {
        d.nodes = (long long)N;
        d.tets = (long long)T;
        d.index = reinterpret_cast<const uint4*>(index);
        d.slot = reinterpret_cast<const uint4*>(slot);
        d.fixed = A.upload(fixed.data(), N);
        d.offset = offset;
        d.counter = A.zeros<long long>(2);
        d.e_diss = A.zeros<double>(s->eblocks);
        d.e_strain = A.zeros<double>(s->eblocks);
        d.n_work = A.zeros<double>(s->nblocks);
        d.n_kin = A.zeros<double>(s->nblocks);
        d.n_grav = A.zeros<double>(s->nblocks);
    };
    if (!rc && mode == FEMSTEP_TET_J2_F64) {
        TetDevice<double>& d = s->d64;
        common(d);
        double* pos = A.alloc<double>(N * 3);
        if (pos) fs::launch_widen(pos32, (long long)N * 3, pos, s->stream);
        d.position = pos;
        std::vector<double> vel(N * 3, 0.0);
        if (m.velocity)
            for (size_t i = 0; i < N * 3; ++i) vel[i] = m.velocity[i];
        d.velocity = A.upload(vel.data(), N * 3);
        d.mass = mass64;
        d.rest_inv = inv64;
        d.rest_vol = vol64;
        d.plastic = A.zeros<double>(T * 7);
        if (m.external_force) d.ext = A.upload(m.external_force, N * 3);
        d.slots = A.zeros<double>(T * 4 * 3 + 2);
    } else if (!rc) {
        TetDevice<float>& d = s->d32;
        common(d);
        std::vector<float> vel(N * 3, 0.0f);
        if (m.velocity) std::memcpy(vel.data(), m.velocity, sizeof(float) * N * 3);
        d.velocity = A.upload(vel.data(), N * 3);
        d.slots = A.zeros<float>(T * 4 * 4 + 4);  // a padded float4 per corner
        s->rest.assign(m.position, m.position + N * 3);
        d.rest = pos32;
        d.disp = A.zeros<float>(N * 4);
        if (mode == FEMSTEP_TET_J2_F32K) d.disp_c = A.zeros<float>(N * 4);
        float* inv32 = A.alloc<float>(T * 9);
        float* vol32 = A.alloc<float>(T);
        float* mass32 = A.alloc<float>(N);
        float* inv_mass32 = A.alloc<float>(N);
        if (A.ok())
            fs::launch_tet_rest_f32(inv64, vol64, (long long)T, mass64, (long long)N, inv32, vol32, mass32, inv_mass32,
                                    s->stream);
        d.rest_inv = inv32;
        d.rest_vol = vol32;
        d.mass = mass32;
        d.inv_mass = inv_mass32;
        d.plastic = A.zeros<float>(T * 7);
        if (mode == FEMSTEP_TET_J2_F32K) d.plastic_c = A.zeros<float>(T * 7);
        if (m.external_force) {
            std::vector<float> ext(N * 3);
            for (size_t i = 0; i < N * 3; ++i) ext[i] = (float)m.external_force[i];
            d.ext = A.upload(ext.data(), N * 3);
        }
        s->inv64 = inv64;
    }
    s->d_out = A.zeros<double>(8);
    if (!rc) rc = check(s, cudaStreamSynchronize(s->stream), "set-up");
    fs::device_free(entry);
    fs::device_free(quarter);
    if (!rc && !A.ok()) {
        const int code = A.status() == cudaErrorMemoryAllocation ? FEMSTEP_ENOMEM : FEMSTEP_ECUDA;
        rc = fail(s, code, std::string("device upload failed: ") + cudaGetErrorString(A.status()));
    }
    if (rc) {
        femstep_tet_destroy(s);
        return rc;
    }
    *out = s;
    return FEMSTEP_OK;
}

}  // namespace

extern "C" {

int femstep_tet_create(const femstep_tet_mesh* mesh, int mode, femstep_tet** out) {
    if (out) *out = nullptr;
    if (!mesh || !out) return fail(nullptr, FEMSTEP_EINVAL, "null mesh or output handle");
    if (mode < FEMSTEP_TET_REF32 || mode > FEMSTEP_TET_J2_F64) return fail(nullptr, FEMSTEP_EINVAL, "unknown mode");
    const femstep_tet_mesh& m = *mesh;
    const size_t N = m.nodes, T = m.tets;
    if (N == 0 || T == 0) return fail(nullptr, FEMSTEP_EINVAL, "empty mesh");
    if (N >= 0xffffffffu || T * 4 >= 0xffffffffu) return fail(nullptr, FEMSTEP_EINVAL, "mesh too large for 32-bit ids");
    if (!m.position || !m.index) return fail(nullptr, FEMSTEP_EINVAL, "position and index are required");
    for (size_t i = 0; i < T * 4; ++i)
        if (m.index[i] >= N) return fail(nullptr, FEMSTEP_EINVAL, "tet index out of range");
    if (mode == FEMSTEP_TET_REF32 && (!m.mass || !m.rest_inv || !m.rest_volume))
        return fail(nullptr, FEMSTEP_EINVAL, "REF32 needs the caller's mass, rest_inv and rest_volume");
    if (mode != FEMSTEP_TET_REF32 && !(m.density > 0.0))
        return fail(nullptr, FEMSTEP_EINVAL, "J2 modes need a positive density");

    // The J2 modes without a caller adjacency are set up on the device: the CSR (the
    // counting sort's order), the slot map and the FP64 rest state.
    if (mode != FEMSTEP_TET_REF32 && !(m.adjacency_offset && m.adjacency_entry)) return create_on_device(m, mode, out);

    // CSR: the caller's (validated), or built by counting sort as fem.cpp:147-157.
    std::vector<uint32_t> offset, entry;
    if (m.adjacency_offset && m.adjacency_entry) {
        offset.assign(m.adjacency_offset, m.adjacency_offset + N + 1);
        entry.assign(m.adjacency_entry, m.adjacency_entry + T * 4);
        if (offset[0] != 0 || offset[N] != T * 4) return fail(nullptr, FEMSTEP_EINVAL, "adjacency offsets do not span 4T entries");
        for (size_t n = 0; n < N; ++n)
            if (offset[n + 1] < offset[n]) return fail(nullptr, FEMSTEP_EINVAL, "adjacency offsets decrease");
    } else {
        fs::build_csr(N, T, 4, m.index, offset, entry);
    }
    std::vector<uint32_t> slot(T * 4, 0xffffffffu);
    for (size_t n = 0; n < N; ++n)
        for (uint32_t k = offset[n]; k < offset[n + 1]; ++k) {
            const uint32_t e = entry[k];
            if (e >= T * 4 || m.index[e] != n || slot[e] != 0xffffffffu)
                return fail(nullptr, FEMSTEP_EINVAL, "adjacency is not the node-to-corner map of this mesh");
            slot[e] = k;
        }
    // The mesh is checked before the device, so a bad mesh is reported as such on any
    // machine; a good one on a machine with no GPU is a skip.
    const int dev = fs::device_status();
    if (dev != FEMSTEP_OK) return dev;

    femstep_tet* s = new femstep_tet();
    s->mode = mode;
    s->nodes = N;
    s->tets = T;
    s->eblocks = fs::blocks_for((long long)T, fs::kBlock);
    s->nblocks = fs::blocks_for((long long)N, fs::kBlock);
    int rc = check(s, cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "stream");
    if (rc == FEMSTEP_OK) rc = check(s, cudaEventCreate(&s->ev0), "event");
    if (rc == FEMSTEP_OK) rc = check(s, cudaEventCreate(&s->ev1), "event");
    if (rc != FEMSTEP_OK) {
        femstep_tet_destroy(s);
        return rc;
    }
    fs::DeviceArena& A = s->arena;
    std::vector<uint8_t> fixed(N, 0);
    if (m.fixed)
        for (size_t n = 0; n < N; ++n) fixed[n] = m.fixed[n] ? 1 : 0;

    std::vector<double> inv64, vol64, mass64;
    if (mode != FEMSTEP_TET_REF32) rest_state64(m, inv64, vol64, mass64);

    auto common = [&](auto& d) {
        d.nodes = (long long)N;
        d.tets = (long long)T;
        d.index = (const uint4*)A.upload(m.index, T * 4);
        d.slot = (const uint4*)A.upload(slot.data(), T * 4);
        d.fixed = A.upload(fixed.data(), N);
        d.offset = A.upload(offset.data(), N + 1);
        d.counter = A.zeros<long long>(2);
        d.e_diss = A.zeros<double>(s->eblocks);
        d.e_strain = A.zeros<double>(s->eblocks);
        d.n_work = A.zeros<double>(s->nblocks);
        d.n_kin = A.zeros<double>(s->nblocks);
        d.n_grav = A.zeros<double>(s->nblocks);
    };

    if (mode == FEMSTEP_TET_J2_F64) {
        TetDevice<double>& d = s->d64;
        common(d);
        std::vector<double> pos(N * 3), vel(N * 3, 0.0);
        for (size_t i = 0; i < N * 3; ++i) pos[i] = m.position[i];
        if (m.velocity)
            for (size_t i = 0; i < N * 3; ++i) vel[i] = m.velocity[i];
        d.position = A.upload(pos.data(), N * 3);
        d.velocity = A.upload(vel.data(), N * 3);
        d.mass = A.upload(mass64.data(), N);
        const std::vector<double> inv_soa = soa(inv64.data(), T, 9);
        d.rest_inv = A.upload(inv_soa.data(), T * 9);
        d.rest_vol = A.upload(vol64.data(), T);
        d.plastic = A.zeros<double>(T * 7);
        if (m.external_force) d.ext = A.upload(m.external_force, N * 3);
        d.slots = A.zeros<double>(T * 4 * 3 + 2);
    } else {
        TetDevice<float>& d = s->d32;
        common(d);
        std::vector<float> vel(N * 3, 0.0f);
        if (m.velocity) std::memcpy(vel.data(), m.velocity, sizeof(float) * N * 3);
        d.velocity = A.upload(vel.data(), N * 3);
        // REF32: three floats per corner (the reference's layout); J2 modes: a padded
        // float4 per corner, one 16-byte store each
        d.slots = A.zeros<float>(mode == FEMSTEP_TET_REF32 ? T * 4 * 3 + 4 : T * 4 * 4 + 4);
        if (mode == FEMSTEP_TET_REF32) {
            d.position = A.upload(m.position, N * 3);
            d.mass = A.upload(m.mass, N);
            const std::vector<float> inv_soa = soa(m.rest_inv, T, 9);
            d.rest_inv = A.upload(inv_soa.data(), T * 9);
            d.rest_vol = A.upload(m.rest_volume, T);
        } else {
            s->rest.assign(m.position, m.position + N * 3);
            d.rest = A.upload(m.position, N * 3);
            d.disp = A.zeros<float>(N * 4);  // one (x, y, z, 0) float4 per node
            if (mode == FEMSTEP_TET_J2_F32K) d.disp_c = A.zeros<float>(N * 4);
            std::vector<float> mass(N), inv_mass(N), inv(T * 9), vol(T);
            for (size_t n = 0; n < N; ++n) {
                mass[n] = (float)mass64[n];
                inv_mass[n] = mass64[n] > 0.0 ? (float)(1.0 / mass64[n]) : 0.0f;
            }
            for (size_t i = 0; i < T * 9; ++i) inv[i] = (float)inv64[i];
            for (size_t t = 0; t < T; ++t) vol[t] = (float)vol64[t];
            d.mass = A.upload(mass.data(), N);
            d.inv_mass = A.upload(inv_mass.data(), N);
            const std::vector<float> inv_soa = soa(inv.data(), T, 9);
            d.rest_inv = A.upload(inv_soa.data(), T * 9);
            d.rest_vol = A.upload(vol.data(), T);
            d.plastic = A.zeros<float>(T * 7);
            if (mode == FEMSTEP_TET_J2_F32K) d.plastic_c = A.zeros<float>(T * 7);
            if (m.external_force) {
                std::vector<float> ext(N * 3);
                for (size_t i = 0; i < N * 3; ++i) ext[i] = (float)m.external_force[i];
                d.ext = A.upload(ext.data(), N * 3);
            }
        }
    }
    if (mode != FEMSTEP_TET_REF32) s->rest_inv64 = std::move(inv64);
    s->d_out = A.zeros<double>(8);
    if (!A.ok()) {
        const int code = A.status() == cudaErrorMemoryAllocation ? FEMSTEP_ENOMEM : FEMSTEP_ECUDA;
        fail(s, code, std::string("device upload failed: ") + cudaGetErrorString(A.status()));
        femstep_tet_destroy(s);
        return code;
    }
    *out = s;
    return FEMSTEP_OK;
}

int femstep_tet_run(femstep_tet* s, int substeps, const femstep_tet_params* params, double* gpu_ms) {
    if (!s || !params) return fail(s, FEMSTEP_EINVAL, "null solver or params");
    if (substeps < 0) return fail(s, FEMSTEP_EINVAL, "negative step count");
    if (!(params->dt > 0.0) || !std::isfinite(params->dt)) return fail(s, FEMSTEP_EINVAL, "dt must be positive");
    const TetParams q = make_params(s, *params);
    s->launches = 0;
    int rc = check(s, cudaEventRecord(s->ev0, s->stream), "event record");
    if (rc) return rc;
    // Whole chunks replay one captured graph of kGraphSteps steps; the rest launch
    // directly.  The graph bakes the parameters in, so it is rebuilt when they change.
    int left = substeps;
    if (left >= kGraphSteps) {
        if (!s->graph || std::memcmp(&s->graph_params, &q, sizeof(q)) != 0) {
            if (s->graph) cudaGraphExecDestroy(s->graph);
            s->graph = nullptr;
            cudaGraph_t g = nullptr;
            rc = check(s, cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "capture");
            if (rc) return rc;
            for (int i = 0; i < kGraphSteps; ++i) launch_step(s, q);
            rc = check(s, cudaStreamEndCapture(s->stream, &g), "capture end");
            if (rc) return rc;
            rc = check(s, cudaGraphInstantiate(&s->graph, g, 0), "graph instantiate");
            cudaGraphDestroy(g);
            if (rc) return rc;
            s->graph_params = q;
        }
        while (left >= kGraphSteps) {
            rc = check(s, cudaGraphLaunch(s->graph, s->stream), "graph launch");
            if (rc) return rc;
            left -= kGraphSteps;
            s->launches += 2 * kGraphSteps;
        }
    }
    for (; left > 0; --left) {
        launch_step(s, q);
        s->launches += 2;
    }
    rc = check(s, cudaGetLastError(), "kernel launch");
    if (rc) return rc;
    rc = check(s, cudaEventRecord(s->ev1, s->stream), "event record");
    if (rc) return rc;
    rc = check(s, cudaEventSynchronize(s->ev1), "step");
    if (rc) return rc;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, s->ev0, s->ev1);
    if (gpu_ms) *gpu_ms = ms;
    return FEMSTEP_OK;
}

}  // extern "C"

namespace {

// The FP32 modes' displacement, 3N doubles: u, or the compensated u - c.
int displacement(femstep_tet* s, std::vector<double>& out) {
    const size_t N = s->nodes;
    std::vector<float> u(N * 4), c;
    int rc = check(s, cudaMemcpy(u.data(), s->d32.disp, N * 16, cudaMemcpyDeviceToHost), "readback");
    if (!rc && s->d32.disp_c) {
        c.resize(N * 4);
        rc = check(s, cudaMemcpy(c.data(), s->d32.disp_c, N * 16, cudaMemcpyDeviceToHost), "readback");
    }
    if (rc) return rc;
    out.resize(N * 3);
    for (size_t n = 0; n < N; ++n)
        for (int k = 0; k < 3; ++k)
            out[n * 3 + k] = (double)u[n * 4 + k] - (c.empty() ? 0.0 : (double)c[n * 4 + k]);
    return FEMSTEP_OK;
}

}  // namespace

extern "C" {

int femstep_tet_readback(femstep_tet* s, float* position, float* velocity) {
    if (!s) return fail(s, FEMSTEP_EINVAL, "null solver");
    const size_t n3 = s->nodes * 3;
    int rc = FEMSTEP_OK;
    if (s->mode == FEMSTEP_TET_J2_F64) {
        std::vector<double> p, v;
        rc = femstep_tet_readback_f64(s, position ? (p.resize(n3), p.data()) : nullptr,
                                      velocity ? (v.resize(n3), v.data()) : nullptr);
        if (rc) return rc;
        if (position)
            for (size_t i = 0; i < n3; ++i) position[i] = (float)p[i];
        if (velocity)
            for (size_t i = 0; i < n3; ++i) velocity[i] = (float)v[i];
        return FEMSTEP_OK;
    }
    if (position) {
        if (s->mode == FEMSTEP_TET_REF32) {
            rc = check(s, cudaMemcpy(position, s->d32.position, n3 * sizeof(float), cudaMemcpyDeviceToHost), "readback");
        } else {
            std::vector<double> u;
            rc = displacement(s, u);
            for (size_t i = 0; i < n3 && !rc; ++i) position[i] = (float)((double)s->rest[i] + u[i]);
        }
        if (rc) return rc;
    }
    if (velocity)
        rc = check(s, cudaMemcpy(velocity, s->d32.velocity, n3 * sizeof(float), cudaMemcpyDeviceToHost), "readback");
    return rc;
}

int femstep_tet_readback_f64(femstep_tet* s, double* position, double* velocity) {
    if (!s) return fail(s, FEMSTEP_EINVAL, "null solver");
    const size_t n3 = s->nodes * 3;
    int rc = FEMSTEP_OK;
    if (s->mode == FEMSTEP_TET_J2_F64) {
        if (position)
            rc = check(s, cudaMemcpy(position, s->d64.position, n3 * sizeof(double), cudaMemcpyDeviceToHost), "readback");
        if (!rc && velocity)
            rc = check(s, cudaMemcpy(velocity, s->d64.velocity, n3 * sizeof(double), cudaMemcpyDeviceToHost), "readback");
        return rc;
    }
    std::vector<float> p(n3), v(n3);
    if (position) {
        if (s->mode == FEMSTEP_TET_REF32) {
            rc = check(s, cudaMemcpy(p.data(), s->d32.position, n3 * sizeof(float), cudaMemcpyDeviceToHost), "readback");
            for (size_t i = 0; i < n3 && !rc; ++i) position[i] = p[i];
        } else {
            std::vector<double> u;
            rc = displacement(s, u);
            for (size_t i = 0; i < n3 && !rc; ++i) position[i] = (double)s->rest[i] + u[i];
        }
        if (rc) return rc;
    }
    if (velocity) {
        rc = check(s, cudaMemcpy(v.data(), s->d32.velocity, n3 * sizeof(float), cudaMemcpyDeviceToHost), "readback");
        for (size_t i = 0; i < n3 && !rc; ++i) velocity[i] = v[i];
    }
    return rc;
}

int femstep_tet_plastic(femstep_tet* s, double* plastic) {
    if (!s || !plastic) return fail(s, FEMSTEP_EINVAL, "null argument");
    const size_t T = s->tets;
    if (s->mode == FEMSTEP_TET_REF32) {
        std::memset(plastic, 0, sizeof(double) * T * 7);
        return FEMSTEP_OK;
    }
    if (s->mode == FEMSTEP_TET_J2_F64) {
        std::vector<double> a(T * 7);
        const int rc = check(s, cudaMemcpy(a.data(), s->d64.plastic, a.size() * sizeof(double), cudaMemcpyDeviceToHost), "readback");
        if (rc) return rc;
        for (size_t t = 0; t < T; ++t)
            for (int k = 0; k < 7; ++k) plastic[t * 7 + k] = a[(size_t)k * T + t];
        return FEMSTEP_OK;
    }
    std::vector<float> a(T * 7);
    const int rc = check(s, cudaMemcpy(a.data(), s->d32.plastic, a.size() * sizeof(float), cudaMemcpyDeviceToHost), "readback");
    if (rc) return rc;
    for (size_t t = 0; t < T; ++t)
        for (int k = 0; k < 7; ++k) plastic[t * 7 + k] = a[(size_t)k * T + t];
    return FEMSTEP_OK;
}

int femstep_tet_energy(femstep_tet* s, double out[5]) {
    if (!s || !out) return fail(s, FEMSTEP_EINVAL, "null argument");
    for (int i = 0; i < 5; ++i) out[i] = 0.0;
    if (s->mode == FEMSTEP_TET_REF32) return FEMSTEP_OK;
    const bool f64 = s->mode == FEMSTEP_TET_J2_F64;
    const double* arrays[5] = {f64 ? s->d64.n_work : s->d32.n_work, f64 ? s->d64.e_diss : s->d32.e_diss,
                               f64 ? s->d64.e_strain : s->d32.e_strain, f64 ? s->d64.n_kin : s->d32.n_kin,
                               f64 ? s->d64.n_grav : s->d32.n_grav};
    const long long counts[5] = {s->nblocks, s->eblocks, s->eblocks, s->nblocks, s->nblocks};
    for (int i = 0; i < 5; ++i) fs::launch_reduce_sum(arrays[i], counts[i], s->d_out + i, s->stream);
    int rc = check(s, cudaGetLastError(), "reduce");
    if (rc) return rc;
    rc = check(s, cudaMemcpyAsync(out, s->d_out, 5 * sizeof(double), cudaMemcpyDeviceToHost, s->stream), "readback");
    if (rc) return rc;
    return check(s, cudaStreamSynchronize(s->stream), "reduce");
}

int femstep_tet_critical_dt(femstep_tet* s, double youngs, double poisson, double density, double safety,
                            double* dt) {
    if (!s || !dt) return fail(s, FEMSTEP_EINVAL, "null argument");
    if (!(density > 0.0)) return fail(s, FEMSTEP_EINVAL, "density must be positive");
    const size_t T = s->tets;
    const double* inv = nullptr;
    double* tmp = nullptr;
    int rc = FEMSTEP_OK;
    if (s->mode == FEMSTEP_TET_J2_F64) {
        inv = s->d64.rest_inv;
    } else if (s->inv64) {
        inv = s->inv64;  // formed on the device at create
    } else {
        std::vector<double> host(T * 9);
        if (s->mode == FEMSTEP_TET_REF32) {
            std::vector<float> f(T * 9);
            rc = check(s, cudaMemcpy(f.data(), s->d32.rest_inv, f.size() * sizeof(float), cudaMemcpyDeviceToHost), "readback");
            if (rc) return rc;
            for (size_t i = 0; i < f.size(); ++i) host[i] = f[i];  // already SoA
        } else {
            const std::vector<double> a = soa(s->rest_inv64.data(), T, 9);
            host = a;
        }
        rc = check(s, fs::device_alloc((void**)&tmp, host.size() * sizeof(double)), "alloc");
        if (rc) return rc;
        rc = check(s, cudaMemcpy(tmp, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice), "upload");
        if (rc) {
            fs::device_free(tmp);
            return rc;
        }
        inv = tmp;
    }
    double* block_max = nullptr;
    rc = check(s, fs::device_alloc((void**)&block_max, sizeof(double) * s->eblocks), "alloc");
    if (!rc) {
        fs::launch_tet_omega2((long long)T, inv, youngs, poisson, density, block_max, s->eblocks, s->stream);
        fs::launch_reduce_max(block_max, s->eblocks, s->d_out + 7, s->stream);
        double w2 = 0.0;
        rc = check(s, cudaMemcpyAsync(&w2, s->d_out + 7, sizeof(double), cudaMemcpyDeviceToHost, s->stream), "readback");
        if (!rc) rc = check(s, cudaStreamSynchronize(s->stream), "critical dt");
        *dt = w2 > 0.0 ? safety * 2.0 / std::sqrt(w2) : 0.0;
    }
    fs::device_free(block_max);
    if (tmp) fs::device_free(tmp);
    return rc;
}

int femstep_tet_profile(femstep_tet* s, int steps, const femstep_tet_params* params, double out[2]) {
    if (!s || !params || !out) return fail(s, FEMSTEP_EINVAL, "null argument");
    if (steps <= 0) return fail(s, FEMSTEP_EINVAL, "steps must be positive");
    const TetParams q = make_params(s, *params);
    std::vector<cudaEvent_t> ev(3 * (size_t)steps, nullptr);
    int rc = FEMSTEP_OK;
    for (auto& e : ev)
        if (!rc) rc = check(s, cudaEventCreate(&e), "event");
    for (int i = 0; i < steps && !rc; ++i) {
        cudaEventRecord(ev[3 * i], s->stream);
        launch_step(s, q, fs::kElementPart);
        cudaEventRecord(ev[3 * i + 1], s->stream);
        launch_step(s, q, fs::kNodePart);
        cudaEventRecord(ev[3 * i + 2], s->stream);
    }
    if (!rc) rc = check(s, cudaGetLastError(), "kernel launch");
    if (!rc) rc = check(s, cudaStreamSynchronize(s->stream), "profile");
    double e_ms = 0.0, n_ms = 0.0;
    for (int i = 0; i < steps && !rc; ++i) {
        float a = 0.0f, b = 0.0f;
        cudaEventElapsedTime(&a, ev[3 * i], ev[3 * i + 1]);
        cudaEventElapsedTime(&b, ev[3 * i + 1], ev[3 * i + 2]);
        e_ms += a;
        n_ms += b;
    }
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    out[0] = e_ms / steps;
    out[1] = n_ms / steps;
    return rc;
}

long long femstep_tet_launches(const femstep_tet* s) { return s ? s->launches : 0; }

const char* femstep_tet_error(const femstep_tet* s) { return s ? s->error.c_str() : fs::last_error(); }

void femstep_tet_destroy(femstep_tet* s) {
    if (!s) return;
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->graph) cudaGraphExecDestroy(s->graph);
    s->arena.release();
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

}  // extern "C"
