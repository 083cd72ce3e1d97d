// api_shell.cu -- host side of the solid-shell zone step behind the C ABI.
//
// Replaces gpu::ZoneGpuSolver (engine/gpu/zone_gpu.{hpp,cpp}): initialise uploads the
// patch (or forms it on the device), run records `substeps` steps without the host in
// the loop, readback returns positions, velocities and the plastic state in the layout
// zone::Solver::adopt consumes.  Errors are a status plus text; no device is a skip.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/femstep.h"
#include "common.cuh"
#include "host_util.hpp"
#include "shell.hpp"
#include "tet.hpp"

using fs::ShellDevice;
using fs::ShellParams;

struct femstep_shell {
    size_t nodes = 0, elements = 0;
    long long groups = 0;
    cudaStream_t stream = nullptr;
    fs::DeviceArena arena;
    ShellDevice d;
    int eblocks = 0, nblocks = 0;
    long long ewarps = 0;             // element-kernel warps = per-warp partial entries
    float* kaa_factor = nullptr;      // [E][32] elastic K_aa factor, for factor_E / factor_nu
    double factor_E = 0.0, factor_nu = 0.0;
    double* d_out = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaGraphExec_t graph = nullptr;
    ShellParams graph_params{};
    long long launches = 0;
    float* fail_strain = nullptr;  // [E] per-element failure strain (+inf: never fails)
    // alpha in double for the EAS64 = 3 variant, allocated on its first run; `alpha64_live`:
    // it holds the current alpha (else the float copy does, and it is reloaded from it)
    bool alpha64_live = false;
    // the punch (femstep_shell_set_punch) and its host-side account, as the reference's
    // GPU zone step keeps it (zone_gpu.cpp:889-919)
    uint8_t* driven = nullptr;     // [N]
    double* n_punch = nullptr;     // [nblocks]
    bool punch = false;
    double punch_speed = 0.0, punch_ramp = 0.0, axis[3] = {0.0, 0.0, 0.0};
    double punch_time = 0.0, punch_penetration = 0.0;
    long long punch_steps = 0;
    // the inertial punch (mass > 0): its state lives on the device
    double punch_mass = 0.0;
    uint32_t* driven_list = nullptr;
    size_t driven_capacity = 0;
    double* punch_state = nullptr;    // [8]
    int* halt = nullptr;
    // the driven edge (femstep_shell_set_edge)
    int* edge_map = nullptr;
    double* edge_rows = nullptr;      // [2][rows][3]: meshed - rest, prescribed
    size_t edge_capacity = 0, edge_dof = 0;
    double edge_ramp = 0.0;
    double* n_edge = nullptr;         // [nblocks]
    // constraint fibres (femstep_shell_set_fibers)
    size_t fiber_capacity = 0;
    int fblocks = 0;
    std::vector<uint8_t> pin;         // host copy of the pinned bits (0-2)
    std::vector<double> rest;  // host copy for readback
    std::string error;
};

namespace {

int fail(femstep_shell* s, int code, const std::string& what) {
    if (s) s->error = what;
    fs::set_last_error(what);
    return code;
}

int check(femstep_shell* s, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return FEMSTEP_OK;
    return fail(s, e == cudaErrorMemoryAllocation ? FEMSTEP_ENOMEM : FEMSTEP_ECUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

ShellParams make_params(const femstep_shell_params& p) {
    ShellParams q{};
    const double E = p.youngs_modulus, nu = p.poisson_ratio;
    // plasticity::Material::shearModulus / bulkModulus (plasticity.hpp:226-227)
    const double mu = E / (2.0 * (1.0 + nu)), kappa = E / (3.0 * (1.0 - 2.0 * nu));
    q.inv_2mu = 1.0 / (2.0 * mu);
    q.inv_3kappa = 1.0 / (3.0 * kappa);
    q.mu = (float)mu;
    q.kappa = (float)kappa;
    q.yield = (float)p.yield_strength;
    q.hardening = (float)p.hardening_modulus;
    q.dt = (float)p.dt;
    q.dt64 = p.dt;
    q.damping = (float)p.damping;
    q.damping64 = p.damping;
    q.rise_time = p.rise_time;
    q.max_iterations = p.max_iterations > 0 ? p.max_iterations : 12;
    // the reference's tolerances (solid_shell.cpp:939, 988) unless the caller gives its own
    q.tol_residual = (float)(p.tol_residual > 0 ? p.tol_residual : 1e-12);
    q.tol_work = (float)(p.tol_work > 0 ? p.tol_work : 1e-16);
    q.compensated = p.compensated;
    q.eas64 = p.eas_fp64;
    // the fibres' law in double: the same material, linear unless the curve is Swift
    q.fiber.youngs = E;
    q.fiber.yield = p.yield_strength;
    q.fiber.hardening = p.hardening_modulus;
    q.fiber.swift = 0;
    q.fiber.tri_sens = 1.5;
    q.fiber.tri_ref = 1.0 / 3.0;
    q.fiber.tri_cut = -1.0 / 3.0;
    if (p.material) {
        const femstep_shell_material& m = *p.material;
        q.fiber.swift = m.hardening == FEMSTEP_SHELL_SWIFT ? 1 : 0;
        q.fiber.swift_k = m.strength_coefficient;
        q.fiber.swift_eps0 = m.reference_strain;
        q.fiber.swift_n = m.hardening_exponent;
        q.fiber.tri_sens = m.triaxiality_sensitivity;
        q.fiber.tri_ref = m.reference_triaxiality;
        q.fiber.tri_cut = m.cutoff_triaxiality;
    }
    if (p.material) {
        const femstep_shell_material& m = *p.material;
        q.general = 1;
        q.swift = m.hardening == FEMSTEP_SHELL_SWIFT ? 1 : 0;
        if (q.swift) q.yield = (float)(m.strength_coefficient * std::pow(m.reference_strain, m.hardening_exponent));
        q.swift_k = (float)m.strength_coefficient;
        q.swift_eps0 = (float)m.reference_strain;
        q.swift_n = (float)m.hardening_exponent;
        q.kinematic = (float)m.kinematic_modulus;
        q.tri_sens = (float)m.triaxiality_sensitivity;
        q.tri_ref = (float)m.reference_triaxiality;
        q.tri_cut = (float)m.cutoff_triaxiality;
    }
    return q;
}

constexpr int kGraphSteps = 16;

// The elastic K_aa factor depends on the material: formed before the first run and
// again whenever E or nu change.
int ensure_factor(femstep_shell* s, const femstep_shell_params& p) {
    if (s->d.kaa_factor && s->factor_E == p.youngs_modulus && s->factor_nu == p.poisson_ratio) return FEMSTEP_OK;
    fs::launch_shell_elastic_factor(s->d, p.youngs_modulus, p.poisson_ratio, s->kaa_factor, s->stream);
    const int rc = check(s, cudaGetLastError(), "elastic factor");
    if (rc) return rc;
    s->d.kaa_factor = s->kaa_factor;
    s->factor_E = p.youngs_modulus;
    s->factor_nu = p.poisson_ratio;
    if (s->graph) {
        cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
    }
    return FEMSTEP_OK;
}

// The caller's RestForms (1505 doubles per element, zone_gpu.cpp:28-34 order) against
// the device's FP64 forms of the same rest positions: every element's Gauss weights,
// and all the values of the first 64 elements, each block (B, G, w, J0^-1) to 1e-9 of
// its largest entry.
int check_caller_forms(femstep_shell* s, const double* forms, const double* weights) {
    const size_t E = s->elements;
    std::vector<double> w(E * 8);
    int rc = check(s, cudaMemcpy(w.data(), weights, w.size() * sizeof(double), cudaMemcpyDeviceToHost), "forms check");
    if (rc) return rc;
    for (size_t e = 0; e < E; ++e)
        for (int gp = 0; gp < 8; ++gp) {
            const double mine = w[e * 8 + gp], theirs = forms[e * 1505 + 1488 + gp];
            if (!(std::fabs(mine - theirs) <= 1e-9 * std::fabs(mine)))
                return fail(s, FEMSTEP_EINVAL,
                            "forms: element " + std::to_string(e) + "'s Gauss weights are not those of its rest positions");
        }
    const size_t n = std::min<size_t>(E, 64);
    double* f64 = nullptr;
    rc = check(s, fs::device_alloc((void**)&f64, n * 1507 * sizeof(double)), "forms check");
    if (rc) return rc;
    fs::ShellSetupArgs a{};
    a.elements = (long long)n;
    a.groups = (long long)((n + 3) / 4);
    a.rest = s->d.rest;
    a.index = s->d.index;
    a.slot = s->d.slot;
    a.formulation = 2;
    a.forms64 = f64;
    fs::launch_shell_setup(a, s->stream);
    std::vector<double> h(n * 1507);
    rc = check(s, cudaMemcpyAsync(h.data(), f64, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream),
               "forms check");
    if (!rc) rc = check(s, cudaStreamSynchronize(s->stream), "forms check");
    fs::device_free(f64);
    if (rc) return rc;
    const size_t block[5] = {0, 1152, 1488, 1496, 1505};
    for (size_t e = 0; e < n; ++e)
        for (int b = 0; b < 4; ++b) {
            const double* mine = h.data() + e * 1507;
            const double* theirs = forms + e * 1505;
            double scale = 0.0;
            for (size_t k = block[b]; k < block[b + 1]; ++k) scale = std::max(scale, std::fabs(mine[k]));
            for (size_t k = block[b]; k < block[b + 1]; ++k)
                if (!(std::fabs(mine[k] - theirs[k]) <= 1e-9 * scale))
                    return fail(s, FEMSTEP_EINVAL,
                                "forms: element " + std::to_string(e) +
                                    "'s forms are not the solid-shell forms of its rest positions");
        }
    return FEMSTEP_OK;
}

}  // namespace

extern "C" {

int femstep_shell_create(const femstep_shell_mesh* mesh, femstep_shell** out) {
    if (out) *out = nullptr;
    if (!mesh || !out) return fail(nullptr, FEMSTEP_EINVAL, "null mesh or output handle");
    const femstep_shell_mesh& m = *mesh;
    const size_t N = m.nodes, E = m.elements;
    if (N == 0 || E == 0) return fail(nullptr, FEMSTEP_EINVAL, "empty mesh");
    if (N >= 0xffffffffu || E * 8 >= 0xffffffffu) return fail(nullptr, FEMSTEP_EINVAL, "mesh too large for 32-bit ids");
    if (!m.rest || !m.index) return fail(nullptr, FEMSTEP_EINVAL, "rest and index are required");
    {
        std::atomic<bool> bad{false};
        fs::parallel_chunks(E * 8, [&](size_t b, size_t e) {
            for (size_t i = b; i < e; ++i)
                if (m.index[i] >= N) {
                    bad = true;
                    return;
                }
        });
        if (bad) return fail(nullptr, FEMSTEP_EINVAL, "element index out of range");
    }
    if (!m.mass && !(m.density > 0.0)) return fail(nullptr, FEMSTEP_EINVAL, "need a lumped mass or a positive density");
    // The adjacency: the caller's (zone::Solver's), checked here on the host together with
    // its slot map; or, without one, built on the device once the index is there
    // (csr.cu: the same runs as the CPU counting sort).
    const bool caller_csr = m.adjacency_offset && m.adjacency_entry;
    std::vector<uint32_t> offset, entry, slot;
    if (caller_csr) {
        offset.assign(m.adjacency_offset, m.adjacency_offset + N + 1);
        entry.assign(m.adjacency_entry, m.adjacency_entry + E * 8);
        if (offset[0] != 0 || offset[N] != E * 8) return fail(nullptr, FEMSTEP_EINVAL, "adjacency offsets do not span 8E entries");
        slot.assign(E * 8, 0xffffffffu);
    }
    // The slot map, node by node: an entry belongs to the one node its corner names, so
    // the nodes' runs touch disjoint slots and run in parallel.
    if (caller_csr) {
        std::atomic<int> bad{0};
        fs::parallel_chunks(N, [&](size_t b, size_t e) {
            for (size_t n = b; n < e && !bad; ++n) {
                if (offset[n + 1] < offset[n]) {
                    bad = 1;
                    return;
                }
                for (uint32_t k = offset[n]; k < offset[n + 1]; ++k) {
                    const uint32_t c = entry[k];
                    if (c >= E * 8 || m.index[c] != n || slot[c] != 0xffffffffu) {
                        bad = 2;
                        return;
                    }
                    slot[c] = k;
                }
            }
        });
        if (bad == 1) return fail(nullptr, FEMSTEP_EINVAL, "adjacency offsets decrease");
        if (bad == 2) return fail(nullptr, FEMSTEP_EINVAL, "adjacency is not the node-to-corner map of this mesh");
    }
    const int dev = fs::device_status();
    if (dev != FEMSTEP_OK) return dev;

    femstep_shell* s = new femstep_shell();
    s->nodes = N;
    s->elements = E;
    s->groups = (long long)((E + 3) / 4);
    s->eblocks = fs::blocks_for(s->groups * 32, fs::kShellBlock);
    s->ewarps = (long long)s->eblocks * (fs::kShellBlock / 32);
    s->nblocks = fs::blocks_for((long long)N, fs::kShellNodeBlock);
    int rc = check(s, cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "stream");
    if (!rc) rc = check(s, cudaEventCreate(&s->ev0), "event");
    if (!rc) rc = check(s, cudaEventCreate(&s->ev1), "event");
    if (rc) {
        femstep_shell_destroy(s);
        return rc;
    }
    fs::DeviceArena& A = s->arena;
    ShellDevice& d = s->d;
    const size_t Epad = (size_t)s->groups * 4;
    d.nodes = (long long)N;
    d.elements = (long long)E;
    d.groups = s->groups;
    {
        int dev = 0, sms = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && sms > 0)
            d.sms = sms;
    }
    s->rest.assign(m.rest, m.rest + N * 3);
    d.rest = A.upload(m.rest, N * 3);
    d.index = A.upload(m.index, E * 8);
    if (caller_csr) {
        d.slot = A.upload(slot.data(), E * 8);
        d.offset = A.upload(offset.data(), N + 1);
    } else {
        uint32_t* dslot = A.alloc<uint32_t>(E * 8);
        uint32_t* doffset = A.alloc<uint32_t>(N + 1);
        d.slot = dslot;
        d.offset = doffset;
        if (A.ok()) {
            rc = check(s, fs::build_csr_device(d.index, (long long)(E * 8), (long long)N, doffset, dslot, s->stream),
                       "adjacency");
            if (rc) {
                femstep_shell_destroy(s);
                return rc;
            }
        }
    }
    float4* elem = A.zeros<float4>(E * fs::kShellElemQ);
    d.elem = elem;
    d.state = A.zeros<float>((size_t)s->groups * fs::kShellStateQ * 32);
    d.alpha = A.zeros<float>(Epad * 8);
    d.state2 = A.zeros<float>((size_t)s->groups * fs::kShellState2Q * 32);
    {
        const std::vector<float> never(E, INFINITY);
        s->fail_strain = A.upload(never.data(), E);
        d.fail_strain = s->fail_strain;
    }
    d.slots = A.zeros<float>(E * 8 * 3 + 4);
    d.counter = A.zeros<long long>(2);
    d.e_diss = A.zeros<double>(s->ewarps);
    d.e_strain = A.zeros<double>(s->ewarps);
    d.e_stats = A.zeros<int>((size_t)s->ewarps * 2);
    s->kaa_factor = A.zeros<float>(E * 32);
    d.n_work = A.zeros<double>(s->nblocks);
    d.n_kin = A.zeros<double>(s->nblocks + 1);  // + the gripped nodes of an inertial punch
    d.punch_kin = d.n_kin + s->nblocks;
    d.n_damp = A.zeros<double>(s->nblocks);
    s->d_out = A.zeros<double>(16);

    // nodes.  The displacement is held as a float u and its Kahan compensation c with
    // position = rest + (u - c): u = fl(x) for the caller's x = position - rest, and c =
    // fl(u - x) carries the part of x that u cannot, so a position read back from this
    // solver (rest + u - c, in double) and handed to a new one continues bit for bit.
    // A node array the caller leaves out starts at zero on the device, not uploaded.
    if (m.position) {
        std::vector<float> disp(N * 3), comp(N * 3);
        fs::parallel_chunks(N * 3, [&](size_t b, size_t e) {
            for (size_t i = b; i < e; ++i) {
                const double x = m.position[i] - m.rest[i];
                disp[i] = (float)x;
                comp[i] = (float)((double)disp[i] - x);
            }
        });
        d.disp = A.upload(disp.data(), N * 3);
        d.disp_c = A.upload(comp.data(), N * 3);
    } else {
        d.disp = A.zeros<float>(N * 3);
        d.disp_c = A.zeros<float>(N * 3);
    }
    if (m.velocity) {
        std::vector<float> vel(N * 3);
        fs::parallel_chunks(N * 3, [&](size_t b, size_t e) {
            for (size_t i = b; i < e; ++i) vel[i] = (float)m.velocity[i];
        });
        d.velocity = A.upload(vel.data(), N * 3);
    } else {
        d.velocity = A.zeros<float>(N * 3);
    }
    std::vector<uint8_t>& pin = s->pin;
    pin.assign(N, 0);
    if (m.pinned)
        fs::parallel_chunks(N, [&](size_t b, size_t e) {
            for (size_t n = b; n < e; ++n)
                pin[n] = (uint8_t)((m.pinned[n * 3] ? 1 : 0) | (m.pinned[n * 3 + 1] ? 2 : 0) |
                                   (m.pinned[n * 3 + 2] ? 4 : 0));
        });
    d.pinned = A.upload(pin.data(), N);
    if (m.load) {
        std::vector<float> load(N * 3);
        fs::parallel_chunks(N * 3, [&](size_t b, size_t e) {
            for (size_t i = b; i < e; ++i) load[i] = (float)m.load[i];
        });
        d.load = A.upload(load.data(), N * 3);
    }
    float* mass = A.alloc<float>(N);
    float* inv_mass = A.alloc<float>(N);
    d.mass = mass;
    d.inv_mass = inv_mass;

    // The element rows (J0^-1, the enhanced modes' scales), and the lumped mass unless
    // the caller gives it, formed here from the rest positions: the step forms B and G
    // from them itself.  Forms handed over by the caller (zone_gpu.cpp:668-684 narrows
    // them for its shaders) must be the solid-shell forms of the same rest positions:
    // every element's Gauss weights, and the whole forms of the first elements, are
    // checked against the device's own FP64 forms.
    double* corner_mass = nullptr;
    double* weights = nullptr;
    if (A.ok()) {
        corner_mass = m.mass ? nullptr : A.zeros<double>(E * 8);
        if (m.forms && fs::device_alloc((void**)&weights, E * 8 * sizeof(double)) != cudaSuccess) {
            femstep_shell_destroy(s);
            return fail(nullptr, FEMSTEP_ENOMEM, "device allocation failed");
        }
        fs::ShellSetupArgs a{};
        a.elements = (long long)E;
        a.groups = s->groups;
        a.rest = d.rest;
        a.index = d.index;
        a.slot = d.slot;
        a.formulation = 2;
        a.density = m.density;
        a.elem = elem;
        a.corner_mass = corner_mass;
        a.gauss_volume = weights;
        fs::launch_shell_setup(a, s->stream);
        if (corner_mass) fs::launch_shell_mass((long long)N, d.offset, corner_mass, nullptr, mass, inv_mass, s->stream);
        cudaStreamSynchronize(s->stream);
        rc = check(s, cudaGetLastError(), "rest forms");
        if (!rc && m.forms) rc = check_caller_forms(s, m.forms, weights);
        if (weights) fs::device_free(weights);
        if (rc) {
            femstep_shell_destroy(s);
            return rc;
        }
    }
    if (A.ok() && m.mass) {
        std::vector<float> mf(N), im(N);
        for (size_t n = 0; n < N; ++n) {
            mf[n] = (float)m.mass[n];
            im[n] = m.mass[n] > 0.0 ? (float)(1.0 / m.mass[n]) : 0.0f;
        }
        cudaMemcpy(mass, mf.data(), N * sizeof(float), cudaMemcpyHostToDevice);
        cudaMemcpy(inv_mass, im.data(), N * sizeof(float), cudaMemcpyHostToDevice);
    }
    if (A.ok() && m.state) {
        // ElementPlasticState (zone_gpu.cpp:36-40): per point plastic strain 0-5, back
        // stress 6-11, eq. plastic strain 12, damage 13, failed 14; enhanced 120-126;
        // failure strain 127; torn 128
        std::vector<float> st((size_t)s->groups * fs::kShellStateQ * 32, 0.0f), al(Epad * 8, 0.0f),
            st2((size_t)s->groups * fs::kShellState2Q * 32, 0.0f), fs_(E);
        for (size_t e = 0; e < E; ++e) {
            const double* x = m.state + e * 129;
            for (int gp = 0; gp < 8; ++gp) {
                const size_t base = (e / 4) * fs::kShellStateQ * 32 + (e % 4) * 8 + gp;
                // plastic strain and eq. plastic strain as a value and its compensation
                // (value - compensation = the caller's double, as for the displacement)
                for (int k = 0; k < 7; ++k) {
                    const double v = x[gp * 15 + (k < 6 ? k : 12)];
                    const float f = (float)v;
                    st[base + (size_t)k * 32] = f;
                    st[base + (size_t)(7 + k) * 32] = (float)((double)f - v);
                }
                const size_t b2 = (e / 4) * fs::kShellState2Q * 32 + (e % 4) * 8 + gp;
                for (int k = 0; k < 6; ++k) st2[b2 + (size_t)k * 32] = (float)x[gp * 15 + 6 + k];
                st2[b2 + (size_t)6 * 32] = (float)x[gp * 15 + 13];
                st2[b2 + (size_t)7 * 32] = x[gp * 15 + 14] != 0.0 ? 1.0f : 0.0f;
            }
            for (int k = 0; k < 7; ++k) al[e * 8 + k] = (float)x[120 + k];
            al[e * 8 + 7] = x[128] != 0.0 ? 1.0f : 0.0f;
            fs_[e] = (float)x[127];
        }
        cudaMemcpy(d.state, st.data(), st.size() * sizeof(float), cudaMemcpyHostToDevice);
        cudaMemcpy(d.alpha, al.data(), al.size() * sizeof(float), cudaMemcpyHostToDevice);
        cudaMemcpy(d.state2, st2.data(), st2.size() * sizeof(float), cudaMemcpyHostToDevice);
        cudaMemcpy(s->fail_strain, fs_.data(), E * sizeof(float), cudaMemcpyHostToDevice);
    }
    if (!A.ok()) {
        const int code = A.status() == cudaErrorMemoryAllocation ? FEMSTEP_ENOMEM : FEMSTEP_ECUDA;
        fail(s, code, std::string("device upload failed: ") + cudaGetErrorString(A.status()));
        femstep_shell_destroy(s);
        return code;
    }
    rc = check(s, cudaDeviceSynchronize(), "upload");
    if (rc) {
        femstep_shell_destroy(s);
        return rc;
    }
    *out = s;
    return FEMSTEP_OK;
}

int femstep_shell_run(femstep_shell* s, int substeps, const femstep_shell_params* params, double* gpu_ms) {
    if (!s || !params) return fail(s, FEMSTEP_EINVAL, "null solver or params");
    if (substeps < 0) return fail(s, FEMSTEP_EINVAL, "negative step count");
    if (!(params->dt > 0.0) || !std::isfinite(params->dt)) return fail(s, FEMSTEP_EINVAL, "dt must be positive");
    if (params->eas_fp64 < 0 || params->eas_fp64 > 3) return fail(s, FEMSTEP_EINVAL, "eas_fp64 must be 0-3");
    if (params->eas_fp64 > 0 && (!params->compensated || !params->material))
        return fail(s, FEMSTEP_EINVAL, "the FP64 enhanced-block variants run the compensated step with a material");
    ShellParams q = make_params(*params);
    if (params->eas_fp64 == 3 && !s->alpha64_live) {
        // alpha into double from its float copy, on this variant's first run
        const size_t n = (size_t)s->groups * 4 * 8;
        if (!s->d.alpha64) {
            s->d.alpha64 = s->arena.alloc<double>(n);
            if (!s->arena.ok()) return fail(s, FEMSTEP_ENOMEM, "alpha in double");
        }
        std::vector<float> af(n);
        std::vector<double> ad(n);
        int rc0 = check(s, cudaMemcpyAsync(af.data(), s->d.alpha, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream),
                        "alpha");
        if (!rc0) rc0 = check(s, cudaStreamSynchronize(s->stream), "alpha");
        for (size_t i = 0; i < n && !rc0; ++i) ad[i] = af[i];
        if (!rc0)
            rc0 = check(s, cudaMemcpyAsync(s->d.alpha64, ad.data(), n * sizeof(double), cudaMemcpyHostToDevice,
                                           s->stream), "alpha");
        if (!rc0) rc0 = check(s, cudaStreamSynchronize(s->stream), "alpha");
        if (rc0) return rc0;
        if (s->graph) {  // a captured graph holds the old device record
            cudaGraphExecDestroy(s->graph);
            s->graph = nullptr;
        }
    }
    s->alpha64_live = params->eas_fp64 == 3;
    q.edge_ramp = s->edge_ramp;
    if (s->punch) {
        q.punch_speed = (float)s->punch_speed;
        q.punch_ramp = s->punch_ramp;
        q.axis_x = (float)s->axis[0];
        q.axis_y = (float)s->axis[1];
        q.axis_z = (float)s->axis[2];
        q.inertial = s->punch_mass > 0.0 ? 1 : 0;
        q.punch_mass = s->punch_mass;
    }
    if (s->punch && !q.inertial) {
        // penetration and time accumulate on the host, step by step, as the reference's
        // GPU zone step does (zone_gpu.cpp:889-919): the speed from the time at the step's start
        for (int k = 0; k < substeps; ++k) {
            const double speed = s->punch_ramp > 0.0 && s->punch_time < s->punch_ramp
                                     ? s->punch_speed * (s->punch_time / s->punch_ramp)
                                     : s->punch_speed;
            s->punch_penetration += speed * params->dt;
            s->punch_time += params->dt;
            ++s->punch_steps;
        }
    }
    s->launches = 0;
    const int per_step = 2 + (q.inertial ? 1 : 0) + (s->d.fibers ? 1 : 0);
    int rc = ensure_factor(s, *params);
    if (rc) return rc;
    rc = check(s, cudaEventRecord(s->ev0, s->stream), "event record");
    if (rc) return rc;
    int left = substeps;
    if (left >= kGraphSteps) {
        if (!s->graph || std::memcmp(&s->graph_params, &q, sizeof(q)) != 0) {
            if (s->graph) cudaGraphExecDestroy(s->graph);
            s->graph = nullptr;
            cudaGraph_t g = nullptr;
            rc = check(s, cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "capture");
            if (rc) return rc;
            for (int i = 0; i < kGraphSteps; ++i) fs::launch_shell_step(s->d, q, s->stream, 3);
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
            s->launches += per_step * kGraphSteps;
        }
    }
    for (; left > 0; --left) {
        fs::launch_shell_step(s->d, q, s->stream, 3);
        s->launches += per_step;
    }
    rc = check(s, cudaGetLastError(), "kernel launch");
    if (!rc) rc = check(s, cudaEventRecord(s->ev1, s->stream), "event record");
    if (!rc) rc = check(s, cudaEventSynchronize(s->ev1), "step");
    if (rc) return rc;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, s->ev0, s->ev1);
    if (gpu_ms) *gpu_ms = ms;
    return FEMSTEP_OK;
}

int femstep_shell_readback(femstep_shell* s, double* position, double* velocity) {
    if (!s) return fail(s, FEMSTEP_EINVAL, "null solver");
    const size_t n3 = s->nodes * 3;
    std::vector<float> buf(n3);
    int rc = FEMSTEP_OK;
    if (position) {
        // the compensated displacement u - c (c stays 0 without compensation)
        std::vector<float> comp(n3);
        rc = check(s, cudaMemcpy(buf.data(), s->d.disp, n3 * sizeof(float), cudaMemcpyDeviceToHost), "readback");
        if (!rc)
            rc = check(s, cudaMemcpy(comp.data(), s->d.disp_c, n3 * sizeof(float), cudaMemcpyDeviceToHost),
                       "readback");
        if (rc) return rc;
        fs::parallel_chunks(n3, [&](size_t b, size_t e) {
            for (size_t i = b; i < e; ++i) position[i] = s->rest[i] + ((double)buf[i] - (double)comp[i]);
        });
    }
    if (velocity) {
        rc = check(s, cudaMemcpy(buf.data(), s->d.velocity, n3 * sizeof(float), cudaMemcpyDeviceToHost), "readback");
        if (rc) return rc;
        fs::parallel_chunks(n3, [&](size_t b, size_t e) {
            for (size_t i = b; i < e; ++i) velocity[i] = buf[i];
        });
    }
    return FEMSTEP_OK;
}

int femstep_shell_set_punch(femstep_shell* s, const uint32_t* driven, size_t count, const double axis[3],
                            double speed, double ramp_time, double mass) {
    if (!s) return fail(s, FEMSTEP_EINVAL, "null solver");
    if (count > 0 && (!driven || !axis)) return fail(s, FEMSTEP_EINVAL, "null argument");
    for (size_t i = 0; i < count; ++i)
        if (driven[i] >= s->nodes) return fail(s, FEMSTEP_EINVAL, "driven node out of range");
    if (count > 0 && !(std::isfinite(speed) && ramp_time >= 0.0)) return fail(s, FEMSTEP_EINVAL, "bad punch speed");
    if (!(mass >= 0.0) || !std::isfinite(mass)) return fail(s, FEMSTEP_EINVAL, "bad punch mass");
    // zone.cpp:779-801: a striking body with no approach speed carries no energy
    if (count > 0 && mass > 0.0 && !(speed > 0.0))
        return fail(s, FEMSTEP_EINVAL, "an inertial punch needs a positive striking mass and approach speed");
    if (!s->driven) {
        s->driven = s->arena.zeros<uint8_t>(s->nodes);
        s->n_punch = s->arena.zeros<double>(s->nblocks);
        s->punch_state = s->arena.zeros<double>(8);
        s->halt = s->arena.zeros<int>(1);
        if (!s->arena.ok()) return check(s, s->arena.status(), "punch allocation");
    }
    std::vector<uint8_t> flag(s->nodes, 0);
    for (size_t i = 0; i < count; ++i) flag[driven[i]] = 1;
    // the list in node order, each node once (the reference's drivenNodes() order)
    std::vector<uint32_t> list;
    for (size_t n = 0; n < s->nodes; ++n)
        if (flag[n]) list.push_back((uint32_t)n);
    if (mass > 0.0 && list.size() > s->driven_capacity) {
        s->driven_list = s->arena.alloc<uint32_t>(list.size());
        if (!s->arena.ok()) return check(s, s->arena.status(), "punch allocation");
        s->driven_capacity = list.size();
    }
    int rc = check(s, cudaMemcpy(s->driven, flag.data(), s->nodes, cudaMemcpyHostToDevice), "punch upload");
    if (!rc) rc = check(s, cudaMemset(s->n_punch, 0, s->nblocks * sizeof(double)), "punch upload");
    const double state0[8] = {mass > 0.0 ? speed : 0.0, 0, 0, 0, 0, 0, 0, 0};
    if (!rc) rc = check(s, cudaMemcpy(s->punch_state, state0, sizeof(state0), cudaMemcpyHostToDevice), "punch upload");
    if (!rc) rc = check(s, cudaMemset(s->halt, 0, sizeof(int)), "punch upload");
    if (!rc) rc = check(s, cudaMemset(s->d.punch_kin, 0, sizeof(double)), "punch upload");
    if (!rc && mass > 0.0 && !list.empty())
        rc = check(s, cudaMemcpy(s->driven_list, list.data(), list.size() * sizeof(uint32_t), cudaMemcpyHostToDevice),
                   "punch upload");
    if (rc) return rc;
    s->punch = count > 0;
    s->punch_mass = s->punch ? mass : 0.0;
    s->d.driven = s->punch ? s->driven : nullptr;
    s->d.n_punch = s->n_punch;
    const bool inertial = s->punch && mass > 0.0;
    s->d.driven_list = inertial ? s->driven_list : nullptr;
    s->d.n_driven = inertial ? (int)list.size() : 0;
    s->d.punch_state = s->punch_state;
    s->d.halt = inertial ? s->halt : nullptr;
    s->punch_speed = speed;
    s->punch_ramp = ramp_time;
    for (int k = 0; k < 3; ++k) s->axis[k] = count > 0 ? axis[k] : 0.0;
    s->punch_time = s->punch_penetration = 0.0;
    s->punch_steps = 0;
    if (s->graph) {  // the graph baked the device layout in
        cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
    }
    return FEMSTEP_OK;
}

int femstep_shell_punch_state(femstep_shell* s, double out[4]) {
    if (!s || !out) return fail(s, FEMSTEP_EINVAL, "null argument");
    out[0] = out[1] = out[2] = out[3] = 0.0;
    if (!s->punch) return FEMSTEP_OK;
    if (s->punch_mass > 0.0) {  // the inertial punch keeps its account on the device
        double st[8];
        const int rc = check(s, cudaMemcpy(st, s->punch_state, sizeof(st), cudaMemcpyDeviceToHost), "readback");
        if (rc) return rc;
        out[0] = st[1];
        out[1] = st[2];
        out[2] = st[3];
        out[3] = st[4];
        return FEMSTEP_OK;
    }
    fs::launch_reduce_sum(s->n_punch, s->nblocks, s->d_out + 4, s->stream);
    int rc = check(s, cudaGetLastError(), "reduce");
    if (!rc) rc = check(s, cudaMemcpyAsync(out, s->d_out + 4, sizeof(double), cudaMemcpyDeviceToHost, s->stream),
                        "readback");
    if (!rc) rc = check(s, cudaStreamSynchronize(s->stream), "reduce");
    if (rc) return rc;
    out[1] = s->punch_penetration;
    out[2] = s->punch_time;
    out[3] = (double)s->punch_steps;
    return FEMSTEP_OK;
}

int femstep_shell_set_edge(femstep_shell* s, const double* prescribed, const double* meshed, double edge_ramp) {
    if (!s) return fail(s, FEMSTEP_EINVAL, "null solver");
    if (!(edge_ramp >= 0.0) || !std::isfinite(edge_ramp)) return fail(s, FEMSTEP_EINVAL, "bad edge ramp");
    const size_t N = s->nodes;
    // zone.cpp:838-840: a pinned DOF with a non-zero prescribed value is driven
    std::vector<uint8_t> pin = s->pin;
    std::vector<int> map(N, -1);
    std::vector<double> base, drive;
    size_t dof = 0;
    for (size_t n = 0; prescribed && n < N; ++n) {
        uint8_t marks = 0;
        for (int k = 0; k < 3; ++k)
            if ((pin[n] & (1u << k)) && prescribed[n * 3 + k] != 0.0) {
                if (!std::isfinite(prescribed[n * 3 + k])) return fail(s, FEMSTEP_EINVAL, "prescribed value not finite");
                marks |= (uint8_t)(8u << k);
            }
        if (!marks) continue;
        map[n] = (int)(base.size() / 3);
        for (int k = 0; k < 3; ++k) {
            const bool on = marks & (8u << k);
            base.push_back(on && meshed ? meshed[n * 3 + k] - s->rest[n * 3 + k] : 0.0);
            drive.push_back(on ? prescribed[n * 3 + k] : 0.0);
            dof += on ? 1 : 0;
        }
        pin[n] |= marks;
    }
    const size_t rows = base.size() / 3;
    fs::DeviceArena& A = s->arena;
    if (rows > 0 && !s->edge_map) {
        s->edge_map = A.alloc<int>(N);
        s->n_edge = A.zeros<double>(s->nblocks);
    }
    if (rows > s->edge_capacity) {
        s->edge_rows = A.alloc<double>(rows * 6);
        s->edge_capacity = rows;
    }
    if (!A.ok()) return check(s, A.status(), "edge allocation");
    int rc = check(s, cudaMemcpy((void*)s->d.pinned, pin.data(), N, cudaMemcpyHostToDevice), "edge upload");
    if (!rc && rows > 0) {
        rc = check(s, cudaMemcpy(s->edge_map, map.data(), N * sizeof(int), cudaMemcpyHostToDevice), "edge upload");
        if (!rc) rc = check(s, cudaMemcpy(s->edge_rows, base.data(), rows * 3 * sizeof(double), cudaMemcpyHostToDevice),
                            "edge upload");
        if (!rc)
            rc = check(s, cudaMemcpy(s->edge_rows + rows * 3, drive.data(), rows * 3 * sizeof(double),
                                     cudaMemcpyHostToDevice),
                       "edge upload");
        if (!rc) rc = check(s, cudaMemset(s->n_edge, 0, s->nblocks * sizeof(double)), "edge upload");
    }
    if (rc) return rc;
    s->d.edge_map = rows > 0 ? s->edge_map : nullptr;
    s->d.edge_base = rows > 0 ? s->edge_rows : nullptr;
    s->d.edge_drive = rows > 0 ? s->edge_rows + rows * 3 : nullptr;
    s->d.n_edge = s->n_edge;
    s->edge_dof = dof;
    s->edge_ramp = edge_ramp;
    if (s->graph) {
        cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
    }
    return FEMSTEP_OK;
}

int femstep_shell_set_fibers(femstep_shell* s, const femstep_shell_fibers* f) {
    if (!s || !f) return fail(s, FEMSTEP_EINVAL, "null argument");
    const size_t F = f->count, N = s->nodes;
    if (F > 0 && (!f->tie || !f->weight || !f->area)) return fail(s, FEMSTEP_EINVAL, "fibre arrays missing");
    if (F >= 0x3fffffffu) return fail(s, FEMSTEP_EINVAL, "too many fibres");
    if (!(f->density >= 0.0)) return fail(s, FEMSTEP_EINVAL, "bad fibre density");
    for (size_t i = 0; i < F * 4; ++i)
        if (f->tie[i] >= N) return fail(s, FEMSTEP_EINVAL, "fibre tie node out of range");
    // rest lengths: the caller's, or from the rest positions as restFibers does
    // (constraint.cpp:185-196)
    std::vector<double> length(F);
    for (size_t i = 0; i < F; ++i) {
        if (f->rest_length) {
            length[i] = f->rest_length[i];
            continue;
        }
        double span[3];
        for (int k = 0; k < 3; ++k) {
            const double* r = s->rest.data();
            const double w0 = f->weight[i * 2], w1 = f->weight[i * 2 + 1];
            const double a = r[(size_t)f->tie[i * 4] * 3 + k] * (1.0 - w0) + r[(size_t)f->tie[i * 4 + 1] * 3 + k] * w0;
            const double b =
                r[(size_t)f->tie[i * 4 + 2] * 3 + k] * (1.0 - w1) + r[(size_t)f->tie[i * 4 + 3] * 3 + k] * w1;
            span[k] = b - a;
        }
        length[i] = std::sqrt(span[0] * span[0] + span[1] * span[1] + span[2] * span[2]);
    }
    std::vector<double> never(F, INFINITY);
    // node -> fibre slot CSR, ascending fibre order per node
    std::vector<uint32_t> offset(N + 1, 0u), entry(F * 4);
    for (size_t i = 0; i < F * 4; ++i) ++offset[f->tie[i] + 1];
    for (size_t n = 0; n < N; ++n) offset[n + 1] += offset[n];
    {
        std::vector<uint32_t> cursor(offset.begin(), offset.end() - 1);
        for (size_t i = 0; i < F * 4; ++i) entry[cursor[f->tie[i]]++] = (uint32_t)i;
    }
    fs::DeviceArena& A = s->arena;
    ShellDevice& d = s->d;
    const int fblocks = F ? fs::blocks_for((long long)F, fs::kShellFiberBlock) : 0;
    if (F > s->fiber_capacity) {
        d.fiber_tie = A.alloc<uint4>(F);
        d.fiber_weight = A.alloc<double2>(F);
        d.fiber_area = A.alloc<double>(F);
        d.fiber_length = A.alloc<double>(F);
        d.fiber_fail = A.alloc<double>(F);
        d.fiber_state = A.alloc<double>(F * 4);
        d.fiber_slots = A.alloc<float>(F * 12);
        d.fiber_entry = A.alloc<uint32_t>(F * 4);
        d.f_diss = A.alloc<double>(fblocks);
        d.f_energy = A.alloc<double>(fblocks);
        s->fiber_capacity = F;
    }
    if (F > 0 && !d.fiber_offset) d.fiber_offset = A.alloc<uint32_t>(N + 1);
    if (!A.ok()) return check(s, A.status(), "fibre allocation");
    int rc = FEMSTEP_OK;
    auto put = [&](const void* dst, const void* src, size_t bytes) {
        if (!rc && bytes) rc = check(s, cudaMemcpy((void*)dst, src, bytes, cudaMemcpyHostToDevice), "fibre upload");
    };
    if (F > 0) {
        put(d.fiber_tie, f->tie, F * sizeof(uint4));
        put(d.fiber_weight, f->weight, F * sizeof(double2));
        put(d.fiber_area, f->area, F * sizeof(double));
        put(d.fiber_length, length.data(), F * sizeof(double));
        put(d.fiber_fail, f->failure_strain ? f->failure_strain : never.data(), F * sizeof(double));
        put(d.fiber_offset, offset.data(), (N + 1) * sizeof(uint32_t));
        put(d.fiber_entry, entry.data(), F * 4 * sizeof(uint32_t));
        if (!rc) rc = check(s, cudaMemset(d.fiber_state, 0, F * 4 * sizeof(double)), "fibre upload");
        if (!rc) rc = check(s, cudaMemset(d.fiber_slots, 0, F * 12 * sizeof(float)), "fibre upload");
        if (!rc) rc = check(s, cudaMemset(d.f_diss, 0, fblocks * sizeof(double)), "fibre upload");
        if (!rc) rc = check(s, cudaMemset(d.f_energy, 0, fblocks * sizeof(double)), "fibre upload");
    }
    // the fibres' mass, a quarter to each tie node in fibre order (lumpFiberMass,
    // constraint.cpp:260-276), when the solver's mass does not hold it yet
    if (!rc && F > 0 && f->density > 0.0) {
        std::vector<float> mf(N);
        rc = check(s, cudaMemcpy(mf.data(), d.mass, N * sizeof(float), cudaMemcpyDeviceToHost), "fibre mass");
        if (!rc) {
            std::vector<double> m(mf.begin(), mf.end());
            for (size_t i = 0; i < F; ++i) {
                if (!(length[i] > 0.0) || !(f->area[i] > 0.0)) continue;
                const double quarter = 0.25 * f->density * f->area[i] * length[i];
                for (int k = 0; k < 4; ++k) m[f->tie[i * 4 + k]] += quarter;
            }
            std::vector<float> im(N);
            for (size_t n = 0; n < N; ++n) {
                mf[n] = (float)m[n];
                im[n] = m[n] > 0.0 ? (float)(1.0 / m[n]) : 0.0f;
            }
            put(d.mass, mf.data(), N * sizeof(float));
            put(d.inv_mass, im.data(), N * sizeof(float));
        }
    }
    if (rc) return rc;
    d.fibers = (long long)F;
    s->fblocks = fblocks;
    if (s->graph) {
        cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
    }
    return FEMSTEP_OK;
}

int femstep_shell_fiber_state(femstep_shell* s, double* out) {
    if (!s || !out) return fail(s, FEMSTEP_EINVAL, "null argument");
    if (!s->d.fibers) return FEMSTEP_OK;
    return check(s, cudaMemcpy(out, s->d.fiber_state, (size_t)s->d.fibers * 4 * sizeof(double), cudaMemcpyDeviceToHost),
                 "readback");
}

int femstep_shell_account(femstep_shell* s, double out[6]) {
    if (!s || !out) return fail(s, FEMSTEP_EINVAL, "null argument");
    for (int i = 0; i < 6; ++i) out[i] = 0.0;
    fs::launch_reduce_sum(s->d.n_damp, s->nblocks, s->d_out + 5, s->stream);
    if (s->n_edge) fs::launch_reduce_sum(s->n_edge, s->nblocks, s->d_out + 6, s->stream);
    double r[2] = {0.0, 0.0};
    int rc = check(s, cudaGetLastError(), "reduce");
    if (!rc) rc = check(s, cudaMemcpyAsync(r, s->d_out + 5, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->stream),
                        "readback");
    if (!rc) rc = check(s, cudaStreamSynchronize(s->stream), "reduce");
    if (rc) return rc;
    out[0] = r[0];
    out[1] = s->n_edge ? r[1] : 0.0;
    if (s->punch && s->punch_mass > 0.0) {
        double st[8];
        int halted = 0;
        rc = check(s, cudaMemcpy(st, s->punch_state, sizeof(st), cudaMemcpyDeviceToHost), "readback");
        if (!rc) rc = check(s, cudaMemcpy(&halted, s->halt, sizeof(int), cudaMemcpyDeviceToHost), "readback");
        if (rc) return rc;
        out[2] = st[0];
        out[3] = 0.5 * s->punch_mass * st[0] * st[0];
        out[4] = halted ? 1.0 : 0.0;
    } else if (s->punch) {
        out[2] = s->punch_ramp > 0.0 && s->punch_time < s->punch_ramp ? s->punch_speed * (s->punch_time / s->punch_ramp)
                                                                      : s->punch_speed;
    }
    out[5] = (double)s->edge_dof;
    return FEMSTEP_OK;
}

int femstep_shell_state(femstep_shell* s, double* state) {
    if (!s || !state) return fail(s, FEMSTEP_EINVAL, "null argument");
    const size_t E = s->elements;
    std::vector<float> st((size_t)s->groups * fs::kShellStateQ * 32), al((size_t)s->groups * 4 * 8),
        st2((size_t)s->groups * fs::kShellState2Q * 32), fs_(E);
    int rc = check(s, cudaMemcpy(st.data(), s->d.state, st.size() * sizeof(float), cudaMemcpyDeviceToHost), "readback");
    if (!rc) rc = check(s, cudaMemcpy(al.data(), s->d.alpha, al.size() * sizeof(float), cudaMemcpyDeviceToHost), "readback");
    if (!rc)
        rc = check(s, cudaMemcpy(st2.data(), s->d.state2, st2.size() * sizeof(float), cudaMemcpyDeviceToHost),
                   "readback");
    if (!rc) rc = check(s, cudaMemcpy(fs_.data(), s->fail_strain, E * sizeof(float), cudaMemcpyDeviceToHost), "readback");
    if (rc) return rc;
    std::vector<double> a64;
    if (s->alpha64_live) {  // the EAS64 = 3 variant keeps alpha in double
        a64.resize(al.size());
        rc = check(s, cudaMemcpy(a64.data(), s->d.alpha64, a64.size() * sizeof(double), cudaMemcpyDeviceToHost),
                   "readback");
        if (rc) return rc;
    }
    for (size_t e = 0; e < E; ++e) {
        double* x = state + e * 129;
        std::fill(x, x + 129, 0.0);
        for (int gp = 0; gp < 8; ++gp) {
            const size_t base = (e / 4) * fs::kShellStateQ * 32 + (e % 4) * 8 + gp;
            // the compensated value (value - compensation; the compensation is 0 when the
            // step ran uncompensated from a state with no compensation)
            for (int k = 0; k < 7; ++k)
                x[gp * 15 + (k < 6 ? k : 12)] = (double)st[base + (size_t)k * 32] - (double)st[base + (size_t)(7 + k) * 32];
            const size_t b2 = (e / 4) * fs::kShellState2Q * 32 + (e % 4) * 8 + gp;
            for (int k = 0; k < 6; ++k) x[gp * 15 + 6 + k] = st2[b2 + (size_t)k * 32];
            x[gp * 15 + 13] = st2[b2 + (size_t)6 * 32];
            x[gp * 15 + 14] = st2[b2 + (size_t)7 * 32];
        }
        for (int k = 0; k < 7; ++k) x[120 + k] = a64.empty() ? (double)al[e * 8 + k] : a64[e * 8 + k];
        x[127] = fs_[e];
        x[128] = al[e * 8 + 7];
    }
    return FEMSTEP_OK;
}

int femstep_shell_energy(femstep_shell* s, double out[4]) {
    if (!s || !out) return fail(s, FEMSTEP_EINVAL, "null argument");
    const double* arrays[4] = {s->d.n_work, s->d.e_diss, s->d.e_strain, s->d.n_kin};
    const long long counts[4] = {s->nblocks, s->ewarps, s->ewarps, s->nblocks + 1};
    for (int i = 0; i < 4; ++i) fs::launch_reduce_sum(arrays[i], counts[i], s->d_out + i, s->stream);
    if (s->d.fibers) {  // the stiffeners' dissipation and strain energy (zone.cpp:1000-1001, 1069)
        fs::launch_reduce_sum(s->d.f_diss, s->fblocks, s->d_out + 8, s->stream);
        fs::launch_reduce_sum(s->d.f_energy, s->fblocks, s->d_out + 9, s->stream);
    }
    double r[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    int rc = check(s, cudaGetLastError(), "reduce");
    if (!rc) rc = check(s, cudaMemcpyAsync(r, s->d_out, sizeof(r), cudaMemcpyDeviceToHost, s->stream), "readback");
    if (!rc) rc = check(s, cudaStreamSynchronize(s->stream), "reduce");
    if (rc) return rc;
    out[0] = r[0];
    out[1] = s->d.fibers ? r[1] + r[8] : r[1];
    out[2] = s->d.fibers ? r[2] + r[9] : r[2];
    out[3] = r[3];
    return FEMSTEP_OK;
}

int femstep_shell_stats(femstep_shell* s, long long out[2]) {
    if (!s || !out) return fail(s, FEMSTEP_EINVAL, "null argument");
    std::vector<int> st((size_t)s->ewarps * 2);
    const int rc = check(s, cudaMemcpy(st.data(), s->d.e_stats, st.size() * sizeof(int), cudaMemcpyDeviceToHost), "readback");
    if (rc) return rc;
    out[0] = out[1] = 0;
    for (long long b = 0; b < s->ewarps; ++b) {
        out[0] += st[b * 2];
        out[1] += st[b * 2 + 1];
    }
    return FEMSTEP_OK;
}

int femstep_shell_critical_dt(femstep_shell* s, double youngs, double poisson, double density, double safety,
                              double* dt) {
    if (!s || !dt) return fail(s, FEMSTEP_EINVAL, "null argument");
    double* per = nullptr;
    int rc = check(s, fs::device_alloc((void**)&per, s->elements * sizeof(double)), "alloc");
    if (rc) return rc;
    fs::ShellSetupArgs a{};
    a.elements = (long long)s->elements;
    a.groups = s->groups;
    a.rest = s->d.rest;
    a.index = s->d.index;
    a.slot = s->d.slot;
    a.formulation = 2;
    a.density = density;
    a.youngs = youngs;
    a.poisson = poisson;
    a.safety = safety;
    a.dt_out = per;
    fs::launch_shell_setup(a, s->stream);
    std::vector<double> h(s->elements);
    rc = check(s, cudaMemcpyAsync(h.data(), per, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream), "readback");
    if (!rc) rc = check(s, cudaStreamSynchronize(s->stream), "critical dt");
    fs::device_free(per);
    if (rc) return rc;
    // smallest positive element step (solid_shell.cpp:1187-1198)
    double best = INFINITY;
    for (double v : h)
        if (v > 0.0) best = std::min(best, v);
    *dt = std::isfinite(best) ? best : 0.0;
    return FEMSTEP_OK;
}

int femstep_shell_profile(femstep_shell* s, int steps, const femstep_shell_params* params, double out[2]) {
    if (!s || !params || !out || steps <= 0) return fail(s, FEMSTEP_EINVAL, "bad argument");
    const ShellParams q = make_params(*params);
    std::vector<cudaEvent_t> ev(3 * (size_t)steps, nullptr);
    int rc = ensure_factor(s, *params);
    for (auto& e : ev)
        if (!rc) rc = check(s, cudaEventCreate(&e), "event");
    for (int i = 0; i < steps && !rc; ++i) {
        cudaEventRecord(ev[3 * i], s->stream);
        fs::launch_shell_step(s->d, q, s->stream, 1);
        cudaEventRecord(ev[3 * i + 1], s->stream);
        fs::launch_shell_step(s->d, q, s->stream, 2);
        cudaEventRecord(ev[3 * i + 2], s->stream);
    }
    if (!rc) rc = check(s, cudaGetLastError(), "kernel launch");
    if (!rc) rc = check(s, cudaStreamSynchronize(s->stream), "profile");
    double a = 0.0, b = 0.0;
    for (int i = 0; i < steps && !rc; ++i) {
        float x = 0.0f, y = 0.0f;
        cudaEventElapsedTime(&x, ev[3 * i], ev[3 * i + 1]);
        cudaEventElapsedTime(&y, ev[3 * i + 1], ev[3 * i + 2]);
        a += x;
        b += y;
    }
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    out[0] = a / steps;
    out[1] = b / steps;
    return rc;
}

long long femstep_shell_launches(const femstep_shell* s) { return s ? s->launches : 0; }
size_t femstep_shell_device_bytes(const femstep_shell* s) { return s ? s->arena.bytes() : 0; }
const char* femstep_shell_error(const femstep_shell* s) { return s ? s->error.c_str() : fs::last_error(); }

// ---- checkpoint / restore ----
//
// The solver's whole mutable state, in a fixed order of device segments after a small
// header: displacement and its compensation, velocity, the element state (plastic
// strain with its compensation, back stress, damage, failed flags, enhanced
// parameters, torn flags), the step counter, every FP64 partial of the energy account
// and the punch, and the host-side punch clock.  What is configuration (mesh, forms,
// mass, the punch's nodes, the driven edge) is not in it: restore into a solver made
// from the same mesh, with the same punch and edge set.  Restoring and running on is
// bit-identical to never having stopped.

namespace {

constexpr uint64_t kShellCheckpointMagic = 0x315048434c485346ull;  // "FSHLCHP1"

struct Segment {
    void* ptr;
    size_t bytes;
};

std::vector<Segment> shell_segments(femstep_shell* s) {
    const size_t N = s->nodes, E = s->elements, Epad = (size_t)s->groups * 4;
    const ShellDevice& d = s->d;
    std::vector<Segment> v = {
        {d.disp, N * 3 * sizeof(float)},
        {d.disp_c, N * 3 * sizeof(float)},
        {d.velocity, N * 3 * sizeof(float)},
        {d.state, (size_t)s->groups * fs::kShellStateQ * 32 * sizeof(float)},
        {d.state2, (size_t)s->groups * fs::kShellState2Q * 32 * sizeof(float)},
        {d.alpha, Epad * 8 * sizeof(float)},
        {d.counter, 2 * sizeof(long long)},
        {d.e_diss, (size_t)s->ewarps * sizeof(double)},
        {d.e_strain, (size_t)s->ewarps * sizeof(double)},
        {d.e_stats, (size_t)s->ewarps * 2 * sizeof(int)},
        {d.n_work, (size_t)s->nblocks * sizeof(double)},
        {d.n_kin, (size_t)(s->nblocks + 1) * sizeof(double)},
        {d.n_damp, (size_t)s->nblocks * sizeof(double)},
    };
    (void)E;
    if (s->driven) {
        v.push_back({s->n_punch, (size_t)s->nblocks * sizeof(double)});
        v.push_back({s->punch_state, 8 * sizeof(double)});
        v.push_back({s->halt, sizeof(int)});
    }
    if (s->n_edge) v.push_back({s->n_edge, (size_t)s->nblocks * sizeof(double)});
    if (d.fibers) {
        v.push_back({d.fiber_state, (size_t)d.fibers * 4 * sizeof(double)});
        v.push_back({d.f_diss, (size_t)s->fblocks * sizeof(double)});
        v.push_back({d.f_energy, (size_t)s->fblocks * sizeof(double)});
    }
    return v;
}

struct CheckpointHeader {
    uint64_t magic;
    uint64_t nodes, elements, segments, payload;
    uint64_t flags;  // 1: punch arrays, 2: edge arrays
    double punch_time, punch_penetration;
    int64_t punch_steps;
};

size_t shell_checkpoint_bytes(femstep_shell* s) {
    size_t total = sizeof(CheckpointHeader);
    for (const Segment& g : shell_segments(s)) total += g.bytes;
    return total;
}

}  // namespace

int femstep_shell_checkpoint_size(femstep_shell* s, size_t* bytes) {
    if (!s || !bytes) return fail(s, FEMSTEP_EINVAL, "null argument");
    *bytes = shell_checkpoint_bytes(s);
    return FEMSTEP_OK;
}

int femstep_shell_checkpoint(femstep_shell* s, void* buffer, size_t bytes) {
    if (!s || !buffer) return fail(s, FEMSTEP_EINVAL, "null argument");
    if (bytes < shell_checkpoint_bytes(s)) return fail(s, FEMSTEP_EINVAL, "checkpoint buffer too small");
    const std::vector<Segment> segs = shell_segments(s);
    CheckpointHeader h{};
    h.magic = kShellCheckpointMagic;
    h.nodes = s->nodes;
    h.elements = s->elements;
    h.segments = segs.size();
    h.payload = shell_checkpoint_bytes(s) - sizeof(h);
    h.flags = (s->driven ? 1u : 0u) | (s->n_edge ? 2u : 0u) | (s->d.fibers ? 4u : 0u);
    h.punch_time = s->punch_time;
    h.punch_penetration = s->punch_penetration;
    h.punch_steps = s->punch_steps;
    int rc = check(s, cudaStreamSynchronize(s->stream), "checkpoint");
    if (rc) return rc;
    char* out = static_cast<char*>(buffer);
    std::memcpy(out, &h, sizeof(h));
    out += sizeof(h);
    for (const Segment& g : segs) {
        rc = check(s, cudaMemcpy(out, g.ptr, g.bytes, cudaMemcpyDeviceToHost), "checkpoint");
        if (rc) return rc;
        out += g.bytes;
    }
    return FEMSTEP_OK;
}

int femstep_shell_restore(femstep_shell* s, const void* buffer, size_t bytes) {
    if (!s || !buffer) return fail(s, FEMSTEP_EINVAL, "null argument");
    if (bytes < sizeof(CheckpointHeader)) return fail(s, FEMSTEP_EINVAL, "not a shell checkpoint");
    CheckpointHeader h;
    std::memcpy(&h, buffer, sizeof(h));
    if (h.magic != kShellCheckpointMagic) return fail(s, FEMSTEP_EINVAL, "not a shell checkpoint");
    if (h.nodes != s->nodes || h.elements != s->elements)
        return fail(s, FEMSTEP_EINVAL, "checkpoint of a different mesh");
    const uint64_t flags = (s->driven ? 1u : 0u) | (s->n_edge ? 2u : 0u) | (s->d.fibers ? 4u : 0u);
    if (h.flags != flags)
        return fail(s, FEMSTEP_EINVAL,
                    "set the punch, the driven edge and the fibres as at the checkpoint before restoring");
    const std::vector<Segment> segs = shell_segments(s);
    if (h.segments != segs.size() || h.payload + sizeof(h) != shell_checkpoint_bytes(s) ||
        bytes < shell_checkpoint_bytes(s))
        return fail(s, FEMSTEP_EINVAL, "checkpoint size does not match this solver");
    int rc = check(s, cudaStreamSynchronize(s->stream), "restore");
    if (rc) return rc;
    const char* in = static_cast<const char*>(buffer) + sizeof(h);
    for (const Segment& g : segs) {
        rc = check(s, cudaMemcpy(g.ptr, in, g.bytes, cudaMemcpyHostToDevice), "restore");
        if (rc) return rc;
        in += g.bytes;
    }
    s->punch_time = h.punch_time;
    s->punch_penetration = h.punch_penetration;
    s->punch_steps = h.punch_steps;
    s->alpha64_live = false;  // the float alpha restored is the current one
    return FEMSTEP_OK;
}

void femstep_shell_destroy(femstep_shell* s) {
    if (!s) return;
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->graph) cudaGraphExecDestroy(s->graph);
    s->arena.release();
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

int femstep_shell_forms(const double* nodes, size_t elements, int formulation, double youngs, double poisson,
                        double density, double safety, double* forms_out, double* mass_out, double* dt_out) {
    if (!nodes || elements == 0) return fail(nullptr, FEMSTEP_EINVAL, "no elements");
    if (formulation < 0 || formulation > 2) return fail(nullptr, FEMSTEP_EINVAL, "unknown formulation");
    const int dev = fs::device_status();
    if (dev != FEMSTEP_OK) return dev;
    fs::DeviceArena A;
    const size_t E = elements;
    std::vector<uint32_t> ident(E * 8);
    for (size_t i = 0; i < E * 8; ++i) ident[i] = (uint32_t)i;
    fs::ShellSetupArgs a{};
    a.elements = (long long)E;
    a.groups = (long long)((E + 3) / 4);
    a.rest = A.upload(nodes, E * 24);
    a.index = A.upload(ident.data(), E * 8);
    a.slot = a.index;
    a.formulation = formulation;
    a.density = density;
    a.youngs = youngs;
    a.poisson = poisson;
    a.safety = safety;
    a.forms64 = forms_out ? A.alloc<double>(E * 1507) : nullptr;
    a.corner_mass = mass_out ? A.alloc<double>(E * 8) : nullptr;
    a.dt_out = dt_out ? A.alloc<double>(E) : nullptr;
    int rc = FEMSTEP_OK;
    if (!A.ok()) {
        rc = fail(nullptr, FEMSTEP_ENOMEM, "device allocation failed");
    } else {
        fs::launch_shell_setup(a, 0);
        cudaError_t e = cudaDeviceSynchronize();
        if (e == cudaSuccess && forms_out) e = cudaMemcpy(forms_out, a.forms64, E * 1507 * sizeof(double), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && mass_out) e = cudaMemcpy(mass_out, a.corner_mass, E * 8 * sizeof(double), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && dt_out) e = cudaMemcpy(dt_out, a.dt_out, E * sizeof(double), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = fail(nullptr, FEMSTEP_ECUDA, std::string("shell forms: ") + cudaGetErrorString(e));
    }
    A.release();
    return rc;
}

}  // extern "C"
