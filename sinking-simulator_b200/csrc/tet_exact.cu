// tet_exact.cu -- the two tet steps that reproduce a CPU path bit for bit.
//
// This translation unit is compiled with -fmad=false: every multiply and add is a
// separately rounded IEEE operation, division and square root are correctly rounded,
// and each expression is written in the order of the CPU code it reproduces.  That is
// what makes these kernels bit-identical to their CPU counterparts:
//
//   REF32  elastic co-rotational tet in float, the arithmetic of fem::tetForces and
//          fem::stepCpu (engine/sim/fem.cpp:73-117, 187-215), i.e. what
//          gpu::FemGpuSolver::run dispatches (engine/gpu/shaders/tet_forces.comp,
//          node_integrate.comp).  Drop-in for the reference's GPU tet back-end.
//   F64    the J2 tet in double: fem.cpp's kinematics with the radial return of
//          plasticity::update (engine/sim/plasticity.cpp:319-505) at the single point,
//          linear isotropic hardening, failure off, and the fem.cpp node update with a
//          ramped external load.  This is the plain FP64 single-mesh step.
//
// Memory-bound kernels (algorithmic bytes: ~240 B per update for REF32, ~435 B for
// F64): one thread per tet / per node, SoA element arrays so each warp load is one
// contiguous 128 B line, node-major force slots so each node's gather is contiguous.
#include "common.cuh"
#include "omega.cuh"
#include "tet.hpp"

namespace fs {
namespace {

// Higham polar iteration.  REF32: four fixed iterations (fem.cpp:62-69).  F64: run to
// convergence, step below 1e-16, at most 64 iterations (solid_shell.cpp:473-487).
__device__ __forceinline__ M3<float> polar_fixed4(const M3<float>& f) {
    M3<float> r = f;
#pragma unroll 1
    for (int i = 0; i < 4; ++i) {
        const M3<float> rit = transpose(inverse(r, 1e-30f));
#pragma unroll
        for (int k = 0; k < 9; ++k) r.m[k] = 0.5f * (r.m[k] + rit.m[k]);
    }
    return r;
}

__device__ __forceinline__ M3<double> polar_converged(const M3<double>& f) {
    M3<double> r = f;
#pragma unroll 1
    for (int it = 0; it < 64; ++it) {
        if (det3(r) == 0.0) return r;
        const M3<double> rit = transpose(inverse(r, 1e-300));
        double worst = 0.0;
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            const double next = 0.5 * (r.m[k] + rit.m[k]);
            const double d = fabs(next - r.m[k]);
            worst = worst > d ? worst : d;
            r.m[k] = next;
        }
        if (worst < 1e-16) return r;
    }
    return r;
}

// ---------------------------------------------------------------------------------
// REF32: fem::tetForces, written to the node-major slots.
__global__ void __launch_bounds__(kBlock) ref32_forces(TetDevice<float> d, float lambda, float mu) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const long long s = d.counter[0];
        d.counter[1] = s;
        d.counter[0] = s + 1;
    }
    if (t >= d.tets) return;
    const uint4 idx = d.index[t];
    const unsigned nid[4] = {idx.x, idx.y, idx.z, idx.w};
    const float* p = d.position;
    M3<float> ds, dm_inv;
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int a = 0; a < 3; ++a) ds(a, c) = p[(size_t)nid[c + 1] * 3 + a] - p[(size_t)nid[0] * 3 + a];
#pragma unroll
    for (int k = 0; k < 9; ++k) dm_inv.m[k] = d.rest_inv[(size_t)k * d.tets + t];
    const M3<float> f = mul(ds, dm_inv);
    const M3<float> r = polar_fixed4(f);
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
    const float scale = -d.rest_vol[t];
    const uint4 sl = d.slot[t];
    const unsigned sid[4] = {sl.x, sl.y, sl.z, sl.w};
    float f0[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float* out = d.slots + (size_t)sid[c + 1] * 3;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float v = scale * h(a, c);
            out[a] = v;
            f0[a] -= v;
        }
    }
    float* out0 = d.slots + (size_t)sid[0] * 3;
#pragma unroll
    for (int a = 0; a < 3; ++a) out0[a] = f0[a];
}

// REF32: fem::stepCpu's node loop (fem.cpp:196-214).
__global__ void __launch_bounds__(kBlock) ref32_nodes(TetDevice<float> d, float dt, float gravity,
                                                      float damping) {
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= d.nodes) return;
    float* vel = d.velocity + (size_t)n * 3;
    if (d.fixed[n]) {
        vel[0] = 0.0f;
        vel[1] = 0.0f;
        vel[2] = 0.0f;
        return;
    }
    const float m = d.mass[n];
    float force[3] = {0.0f, 0.0f, -gravity * m};
    const uint32_t b = d.offset[n], e = d.offset[n + 1];
    const float* sl = d.slots + (size_t)b * 3;
#pragma unroll 4
    for (uint32_t k = b; k < e; ++k, sl += 3) {
        force[0] += sl[0];
        force[1] += sl[1];
        force[2] += sl[2];
    }
    const float inv_mass = 1.0f / m;
    float* pos = d.position + (size_t)n * 3;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float v = vel[k] + force[k] * inv_mass * dt;
        v *= damping;
        vel[k] = v;
        pos[k] += v * dt;
    }
}

// ---------------------------------------------------------------------------------
// F64: the J2 tet.

// plasticity::update for linear isotropic hardening with no kinematic hardening and
// no failure (plasticity.cpp:333-456): elastic predictor, radial return with the
// bracketed Newton on the consistency condition, the committed plastic strain.  The
// arithmetic order is the CPU's, term for term.
struct J2Out {
    double dissipation;
};

__device__ __forceinline__ J2Out j2_return_f64(const double strain[6], double ps[7], double mu, double kappa,
                                               double yield, double hardening, double stress[6]) {
    J2Out out{0.0};
    const double root23 = sqrt(2.0 / 3.0);
    double elastic[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) elastic[i] = strain[i] - ps[i];
    const double volumetric = elastic[0] + elastic[1] + elastic[2];
    const double pressure = kappa * volumetric;
    double trial[6];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        trial[i] = 2.0 * mu * (elastic[i] - volumetric / 3.0);
        trial[3 + i] = mu * elastic[3 + i];
    }
    double relative[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) relative[i] = trial[i] - 0.0;
    const double norm2 = relative[0] * relative[0] + relative[1] * relative[1] + relative[2] * relative[2] +
                         2.0 * (relative[3] * relative[3] + relative[4] * relative[4] + relative[5] * relative[5]);
    const double relative_norm = sqrt(norm2);
    const double pp0 = ps[6] > 0.0 ? ps[6] : 0.0;
    const double yield_radius = root23 * (yield + hardening * pp0);
    const double excess = relative_norm - yield_radius;
    if (!(excess > 0.0)) {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            stress[i] = pressure + trial[i];
            stress[3 + i] = trial[3 + i];
        }
        return out;
    }
    const double linear_part = 2.0 * mu + (2.0 / 3.0) * 0.0;
    double lo = 0.0, hi = excess / linear_part;
    double gamma = hi;
#pragma unroll 1
    for (int iterations = 0; iterations < 50; ++iterations) {
        const double accumulated = ps[6] + root23 * gamma;
        const double pa = accumulated > 0.0 ? accumulated : 0.0;
        const double residual = relative_norm - linear_part * gamma - root23 * (yield + hardening * pa);
        if (residual > 0.0)
            lo = gamma;
        else
            hi = gamma;
        if (fabs(residual) <= 1e-14 * yield_radius) break;
        const double slope = -linear_part - (2.0 / 3.0) * hardening;
        double next = gamma - residual / slope;
        if (!(next > lo && next < hi)) next = 0.5 * (lo + hi);
        if (fabs(next - gamma) <= 1e-15 * gamma) {
            gamma = next;
            break;
        }
        gamma = next;
    }
    double direction[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) direction[i] = relative[i] / relative_norm;
    double dp[6];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        dp[i] = gamma * direction[i];
        dp[3 + i] = 2.0 * gamma * direction[3 + i];
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        stress[i] = pressure + trial[i] - 2.0 * mu * gamma * direction[i];
        stress[3 + i] = trial[3 + i] - 2.0 * mu * gamma * direction[3 + i];
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 6; ++i) s += (stress[i] - (0.0 + (2.0 / 3.0) * 0.0 * gamma * direction[i])) * dp[i];
    out.dissipation = s;
#pragma unroll
    for (int i = 0; i < 6; ++i) ps[i] += dp[i];
    ps[6] += root23 * gamma;
    return out;
}

__global__ void __launch_bounds__(kBlock) f64_forces(TetDevice<double> d, TetParams p) {
    __shared__ double scratch[32];
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const long long s = d.counter[0];
        d.counter[1] = s;
        d.counter[0] = s + 1;
    }
    double diss = 0.0, energy = 0.0;
    if (t < d.tets) {
        const uint4 idx = d.index[t];
        const unsigned nid[4] = {idx.x, idx.y, idx.z, idx.w};
        const double* x = d.position;
        M3<double> ds, dm_inv;
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int a = 0; a < 3; ++a) ds(a, c) = x[(size_t)nid[c + 1] * 3 + a] - x[(size_t)nid[0] * 3 + a];
#pragma unroll
        for (int k = 0; k < 9; ++k) dm_inv.m[k] = d.rest_inv[(size_t)k * d.tets + t];
        const M3<double> f = mul(ds, dm_inv);
        const M3<double> r = polar_converged(f);
        const M3<double> sm = mul(transpose(r), f);
        double strain[6];
        strain[0] = 0.5 * (sm(0, 0) + sm(0, 0)) - 1.0;
        strain[1] = 0.5 * (sm(1, 1) + sm(1, 1)) - 1.0;
        strain[2] = 0.5 * (sm(2, 2) + sm(2, 2)) - 1.0;
        strain[3] = 2.0 * (0.5 * (sm(0, 1) + sm(1, 0)));
        strain[4] = 2.0 * (0.5 * (sm(1, 2) + sm(2, 1)));
        strain[5] = 2.0 * (0.5 * (sm(2, 0) + sm(0, 2)));
        double ps[7];
#pragma unroll
        for (int i = 0; i < 7; ++i) ps[i] = d.plastic[(size_t)i * d.tets + t];
        double sv[6];
        const J2Out j = j2_return_f64(strain, ps, p.mu, p.bulk, p.yield, p.hardening, sv);
#pragma unroll
        for (int i = 0; i < 7; ++i) d.plastic[(size_t)i * d.tets + t] = ps[i];
        const double vol = d.rest_vol[t];
        diss = vol * j.dissipation;
        const double pressure = (sv[0] + sv[1] + sv[2]) / 3.0;
        double density = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i)
            density += 0.5 * sv[i] * ((sv[i] - pressure) / (2.0 * p.mu) + pressure / (3.0 * p.bulk));
#pragma unroll
        for (int i = 3; i < 6; ++i) density += 0.5 * sv[i] * (sv[i] / p.mu);
        energy = vol * density;

        M3<double> stress;
        stress(0, 0) = sv[0];
        stress(1, 1) = sv[1];
        stress(2, 2) = sv[2];
        stress(0, 1) = stress(1, 0) = sv[3];
        stress(1, 2) = stress(2, 1) = sv[4];
        stress(2, 0) = stress(0, 2) = sv[5];
        const M3<double> h = mul(mul(r, stress), transpose(dm_inv));
        const double scale = -vol;
        const uint4 sl = d.slot[t];
        const unsigned sid[4] = {sl.x, sl.y, sl.z, sl.w};
        double f0[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double* out = d.slots + (size_t)sid[c + 1] * 3;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const double v = scale * h(a, c);
                out[a] = v;
                f0[a] -= v;
            }
        }
        double* out0 = d.slots + (size_t)sid[0] * 3;
#pragma unroll
        for (int a = 0; a < 3; ++a) out0[a] = f0[a];
    }
    const double bd = block_sum(diss, scratch);
    const double be = block_sum(energy, scratch);
    if (threadIdx.x == 0) {
        d.e_diss[blockIdx.x] += bd;
        d.e_strain[blockIdx.x] = be;
    }
}

__global__ void __launch_bounds__(kBlock) f64_nodes(TetDevice<double> d, TetParams p) {
    __shared__ double scratch[32];
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double work = 0.0, kin = 0.0, gwork = 0.0;
    if (n < d.nodes) {
        double* vel = d.velocity + (size_t)n * 3;
        if (d.fixed[n]) {
            vel[0] = 0.0;
            vel[1] = 0.0;
            vel[2] = 0.0;
        } else {
            const double lf = ramp_factor(d.counter[1], p.ramp);
            const double m = d.mass[n];
            double force[3] = {0.0, 0.0, -p.gravity * m};
            const uint32_t b = d.offset[n], e = d.offset[n + 1];
            const double* sl = d.slots + (size_t)b * 3;
#pragma unroll 4
            for (uint32_t k = b; k < e; ++k, sl += 3) {
                force[0] += sl[0];
                force[1] += sl[1];
                force[2] += sl[2];
            }
            double ext[3] = {0.0, 0.0, 0.0};
            if (d.ext) {
#pragma unroll
                for (int k = 0; k < 3; ++k) ext[k] = lf * d.ext[(size_t)n * 3 + k];
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) force[k] += ext[k];
            const double inv_mass = 1.0 / m;
            double* pos = d.position + (size_t)n * 3;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                double v = vel[k] + force[k] * inv_mass * p.dt;
                v *= p.damping;
                vel[k] = v;
                pos[k] += v * p.dt;
                work += ext[k] * v * p.dt;
                kin += 0.5 * m * v * v;
            }
            gwork = -p.gravity * m * vel[2] * p.dt;
        }
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

// ---------------------------------------------------------------------------------
// FP64 critical time step: per tet, the largest omega^2 of the lumped-mass element
// (4/rho) lambda_max(B^T C B) by power iteration, as solid_shell.cpp:1088-1133 does
// for the hex (Rayleigh quotient, at most 400 iterations, relative 1e-10, the same
// start vector).  max over elements bounds the assembled problem.
// Dm^-1 may be the FP64 array (single-mesh J2 step) or a pool's FP32 array, read
// from `first` with SoA stride `stride` and promoted to double.
template <typename In>
__global__ void __launch_bounds__(kBlock) tet_omega2(long long tets, const In* rest_inv, long long stride,
                                                     double lambda, double mu, double rho, double* block_max) {
    __shared__ double smax[kBlock];
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double w2 = 0.0;
    if (t < tets) {
        double g[4][3];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int a = 0; a < 3; ++a) g[c + 1][a] = (double)rest_inv[(size_t)(a * 3 + c) * stride + t];
#pragma unroll
        for (int a = 0; a < 3; ++a) g[0][a] = -(g[1][a] + g[2][a] + g[3][a]);
        w2 = tet_omega2_one(g, lambda, mu, rho);
    }
    smax[threadIdx.x] = w2;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) block_max[blockIdx.x] = smax[0];
}

__global__ void __launch_bounds__(1024) reduce_sum(const double* in, long long n, double* out) {
    __shared__ double scratch[32];
    double s = 0.0;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) s += in[i];
    const double total = block_sum(s, scratch);
    if (threadIdx.x == 0) out[0] = total;
}

__global__ void __launch_bounds__(1024) reduce_max(const double* in, long long n, double* out) {
    __shared__ double smax[1024];
    double s = 0.0;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) s = fmax(s, in[i]);
    smax[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = smax[0];
}

// computeRestState (fem.cpp:119-158) in FP64 on the device, with the host's operations
// in the host's order (tet_rest_state64 in api_common.cu, compiled without contraction
// as this file is): per tet Dm^-1 (SoA rows of `tets`), |det| / 6 and its quarter of
// the lumped mass.
__global__ void tet_rest64_kernel(const float* position, const uint32_t* index, long long tets, double density,
                                  double* inv, double* vol, double* quarter) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tets) return;
    const uint32_t* idx = index + t * 4;
    double a[9];  // column-major
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r)
            a[c * 3 + r] = (double)position[(size_t)idx[c + 1] * 3 + r] - (double)position[(size_t)idx[0] * 3 + r];
#define A(r, c) a[(c) * 3 + (r)]
    const double det = A(0, 0) * (A(1, 1) * A(2, 2) - A(1, 2) * A(2, 1)) -
                       A(0, 1) * (A(1, 0) * A(2, 2) - A(1, 2) * A(2, 0)) +
                       A(0, 2) * (A(1, 0) * A(2, 1) - A(1, 1) * A(2, 0));
    const double volume = fabs(det / 6.0);
    const double id = fabs(det) > 1e-300 ? 1.0 / det : 0.0;
    double r[9];
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
    for (int k = 0; k < 9; ++k) inv[(size_t)k * tets + t] = r[k];
    vol[t] = volume;
    quarter[t] = density * volume * 0.25;
}

// Each node's lumped mass: its tets' quarters summed over its CSR run, which lists its
// corners in ascending tet order -- the order the host's loop adds them in.
__global__ void tet_mass64_kernel(const uint32_t* offset, const uint32_t* entry, long long nodes, const double* quarter,
                                  double* mass) {
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nodes) return;
    double m = 0.0;
    for (uint32_t k = offset[n]; k < offset[n + 1]; ++k) m += quarter[entry[k] >> 2];
    mass[n] = m;
}

// The FP32 modes' copies of the FP64 rest state, rounded once.
__global__ void tet_rest_f32_kernel(const double* inv, const double* vol, long long tets, float* inv32, float* vol32) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tets) return;
    for (int k = 0; k < 9; ++k) inv32[(size_t)k * tets + t] = (float)inv[(size_t)k * tets + t];
    vol32[t] = (float)vol[t];
}

__global__ void tet_mass_f32_kernel(const double* mass, long long nodes, float* mass32, float* inv_mass32) {
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nodes) return;
    mass32[n] = (float)mass[n];
    inv_mass32[n] = mass[n] > 0.0 ? (float)(1.0 / mass[n]) : 0.0f;
}

__global__ void widen_kernel(const float* in, long long n, double* out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (double)in[i];
}

}  // namespace

void launch_tet_rest64(const float* position, const uint32_t* index, long long tets, double density, double* inv,
                       double* vol, double* quarter, cudaStream_t stream) {
    tet_rest64_kernel<<<blocks_for(tets, kBlock), kBlock, 0, stream>>>(position, index, tets, density, inv, vol,
                                                                       quarter);
}

void launch_tet_mass64(const uint32_t* offset, const uint32_t* entry, long long nodes, const double* quarter,
                       double* mass, cudaStream_t stream) {
    tet_mass64_kernel<<<blocks_for(nodes, kBlock), kBlock, 0, stream>>>(offset, entry, nodes, quarter, mass);
}

void launch_tet_rest_f32(const double* inv, const double* vol, long long tets, const double* mass, long long nodes,
                         float* inv32, float* vol32, float* mass32, float* inv_mass32, cudaStream_t stream) {
    tet_rest_f32_kernel<<<blocks_for(tets, kBlock), kBlock, 0, stream>>>(inv, vol, tets, inv32, vol32);
    tet_mass_f32_kernel<<<blocks_for(nodes, kBlock), kBlock, 0, stream>>>(mass, nodes, mass32, inv_mass32);
}

void launch_widen(const float* in, long long n, double* out, cudaStream_t stream) {
    widen_kernel<<<blocks_for(n, kBlock), kBlock, 0, stream>>>(in, n, out);
}

void launch_ref32_step(const TetDevice<float>& d, const TetParams& p, cudaStream_t stream, int parts) {
    const float lambda = (float)p.lambda, mu = (float)p.mu;
    if (parts & kElementPart) ref32_forces<<<blocks_for(d.tets, kBlock), kBlock, 0, stream>>>(d, lambda, mu);
    if (parts & kNodePart)
        ref32_nodes<<<blocks_for(d.nodes, kBlock), kBlock, 0, stream>>>(d, (float)p.dt, (float)p.gravity,
                                                                         (float)p.damping);
}

void launch_f64_step(const TetDevice<double>& d, const TetParams& p, cudaStream_t stream, int parts) {
    if (parts & kElementPart) f64_forces<<<blocks_for(d.tets, kBlock), kBlock, 0, stream>>>(d, p);
    if (parts & kNodePart) f64_nodes<<<blocks_for(d.nodes, kBlock), kBlock, 0, stream>>>(d, p);
}

void launch_tet_omega2(long long tets, const double* rest_inv, double E, double nu, double rho,
                       double* per_block_max, int blocks, cudaStream_t stream) {
    const double lambda = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double mu = E / (2.0 * (1.0 + nu));
    tet_omega2<double><<<blocks, kBlock, 0, stream>>>(tets, rest_inv, tets, lambda, mu, rho, per_block_max);
}

void launch_tet_omega2_f32(long long tets, const float* rest_inv, long long stride, double E, double nu, double rho,
                           double* per_block_max, int blocks, cudaStream_t stream) {
    const double lambda = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double mu = E / (2.0 * (1.0 + nu));
    tet_omega2<float><<<blocks, kBlock, 0, stream>>>(tets, rest_inv, stride, lambda, mu, rho, per_block_max);
}

void launch_reduce_sum(const double* in, long long n, double* out, cudaStream_t stream) {
    reduce_sum<<<1, 1024, 0, stream>>>(in, n, out);
}

void launch_reduce_max(const double* in, long long n, double* out, cudaStream_t stream) {
    reduce_max<<<1, 1024, 0, stream>>>(in, n, out);
}

}  // namespace fs
