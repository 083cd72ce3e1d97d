// shell_step.cu -- the solid-shell explicit step in FP32: element kernel and node kernel.
//
// Element kernel: the elastoplastic update of solidshell::elementPlasticUpdate with
// cached forms (engine/sim/solid_shell.cpp:826-1029), one element per 8 lanes, lane g
// owning Gauss point g.  Per element and step:
//
//   1. rotation from the centre deformation gradient (solid_shell.cpp:702, 473): F =
//      I + H with H = (sum_a dN_a(0) (x) d_a) J0^-1; R = I + Q by the Higham iteration
//      carried in the deviation Q (Q <- (Q - (M Q)^T)/2, M = (I + Q)^-1), so no digit of
//      a small rotation is lost to the identity;
//   2. co-rotated displacement relative to corner 0 (B annihilates a translation):
//      u'_a = R^T (dX_a + dd_a) - dX_a = Q^T dX_a + dd_a + Q^T dd_a;
//   3. strain at the lane's point eps_u = B_g u', with B_g formed in the kernel from
//      the element's rest corners (shell_geom.cuh);
//   4. EAS Newton on r(alpha) = sum_g w_g G_g^T sigma_g = 0: every iterate restarts
//      the point law from the step's start state (plasticity.cpp:319-505, linear
//      isotropic hardening), the residual and K_aa = sum_g w_g G_g^T C_g G_g are warp
//      butterfly sums over the element's 8 lanes (fixed order, identical bits in every
//      lane), and each lane runs the same 7x7 Cholesky (solid_shell.cpp:432);
//      convergence on ||r|| or on the correction's energy |delta . r| against
//      sigma_y V with the reference's tolerances (solid_shell.cpp:939, 963-988), or on
//      ||r|| at FP32's rounding floor, with an iteration cap;
//   5. commit the state of the last evaluation, f = -R sum_g w_g B_g^T sigma_g: a
//      3-round reduce-scatter leaves node a's force in lane a, which writes it to the
//      node-major CSR slot.
//
// FP64 only for the per-block energy partials.
#include "common.cuh"
#include "shell.hpp"
#include "shell_geom.cuh"

namespace fs {
namespace {

// The EAS residual's rounding floor in FP32, relative to the magnitude of its terms:
// sixteen ulps of 1.
constexpr float kResidualFloor = 16.0f * 1.1920929e-7f;

__device__ __forceinline__ float sum8(float v) {
    v += __shfl_xor_sync(0xffffffffu, v, 1);
    v += __shfl_xor_sync(0xffffffffu, v, 2);
    v += __shfl_xor_sync(0xffffffffu, v, 4);
    return v;
}

__device__ __forceinline__ double sum8d(double v) {
    v += __shfl_xor_sync(0xffffffffu, v, 1);
    v += __shfl_xor_sync(0xffffffffu, v, 2);
    v += __shfl_xor_sync(0xffffffffu, v, 4);
    return v;
}

// The enhanced strain with alpha in double: the enhanced part summed in double, then
// added to the compatible strain and rounded once.
__device__ __forceinline__ void shell_enhanced_apply64(const float T[24], const float gc[7], const double alpha[7],
                                                       const float base[6], float out[6]) {
    const double b0 = (double)gc[0] * alpha[0], b1 = (double)gc[1] * alpha[1];
    const double b2 = (double)gc[2] * alpha[2] + (double)gc[3] * alpha[3] + (double)gc[4] * alpha[4];
    const double b3 = (double)gc[5] * alpha[5] + (double)gc[6] * alpha[6];
#pragma unroll
    for (int i = 0; i < 6; ++i)
        out[i] = (float)((double)base[i] + (double)T[i] * b0 + (double)T[6 + i] * b1 + (double)T[12 + i] * b2 +
                         (double)T[18 + i] * b3);
}

__device__ __forceinline__ void kahan_add(float& sum, float& comp, float x) {
    const float y = x - comp;
    const float t = sum + y;
    comp = (t - sum) - y;
    sum = t;
}

// Element e's rest corners for the element operators: the bottom corners relative to
// corner 0 and the directors D_c = X_{c+4} - X_c, each difference taken in double and
// rounded once (the same values the step forms from its own node loads).
__device__ __forceinline__ void shell_rest_corners(const ShellDevice& d, long long e, float Xb[4][3], float D[4][3]) {
    const uint4 i0 = reinterpret_cast<const uint4*>(d.index)[e * 2];
    const uint4 i1 = reinterpret_cast<const uint4*>(d.index)[e * 2 + 1];
    const unsigned nid[8] = {i0.x, i0.y, i0.z, i0.w, i1.x, i1.y, i1.z, i1.w};
    const double X0 = d.rest[(size_t)nid[0] * 3], Y0 = d.rest[(size_t)nid[0] * 3 + 1], Z0 = d.rest[(size_t)nid[0] * 3 + 2];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const size_t ob = (size_t)nid[c] * 3, ot = (size_t)nid[c + 4] * 3;
        const double bx = d.rest[ob], by = d.rest[ob + 1], bz = d.rest[ob + 2];
        Xb[c][0] = (float)(bx - X0);
        Xb[c][1] = (float)(by - Y0);
        Xb[c][2] = (float)(bz - Z0);
        D[c][0] = (float)(d.rest[ot] - bx);
        D[c][1] = (float)(d.rest[ot + 1] - by);
        D[c][2] = (float)(d.rest[ot + 2] - bz);
    }
}

// 3x3 row-major inverse with the reference's singular guard
__device__ __forceinline__ void inv3f(const float a[9], float r[9]) {
    const float det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                      a[2] * (a[3] * a[7] - a[4] * a[6]);
    const float id = fabsf(det) > 1e-30f ? 1.0f / det : 0.0f;
    r[0] = (a[4] * a[8] - a[5] * a[7]) * id;
    r[1] = (a[2] * a[7] - a[1] * a[8]) * id;
    r[2] = (a[1] * a[5] - a[2] * a[4]) * id;
    r[3] = (a[5] * a[6] - a[3] * a[8]) * id;
    r[4] = (a[0] * a[8] - a[2] * a[6]) * id;
    r[5] = (a[2] * a[3] - a[0] * a[5]) * id;
    r[6] = (a[3] * a[7] - a[4] * a[6]) * id;
    r[7] = (a[1] * a[6] - a[0] * a[7]) * id;
    r[8] = (a[0] * a[4] - a[1] * a[3]) * id;
}

struct PointOut {
    float sigma[6];
    float n[6];        // flow direction (tensor components), valid when yielded
    float theta, theta_bar;
    float dp[6];       // plastic strain increment (engineering shears)
    float deq;
    bool yielded;
    // the general point law's trial state
    float back[6];     // back stress after the increment
    float damage;
    bool failed;       // failed (stress and tangent zero)
    float diss;        // dissipation density (sigma - back) : d(eps_p)
};

// Radial return, linear isotropic hardening, no back stress, failure off
// (plasticity.cpp:333-456) with the algorithmic tangent's scalars (:490-504).
__device__ __forceinline__ void point_law(const float eps[6], const float ps[7], const ShellParams& p, PointOut& o) {
    float el[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) el[i] = eps[i] - ps[i];
    const float vol = el[0] + el[1] + el[2];
    const float pressure = p.kappa * vol;
    float trial[6];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        trial[i] = 2.0f * p.mu * (el[i] - vol * (1.0f / 3.0f));
        trial[3 + i] = p.mu * el[3 + i];
    }
    const float norm = sqrtf(trial[0] * trial[0] + trial[1] * trial[1] + trial[2] * trial[2] +
                             2.0f * (trial[3] * trial[3] + trial[4] * trial[4] + trial[5] * trial[5]));
    const float root23 = 0.81649658092772603f;
    const float radius = root23 * (p.yield + p.hardening * fmaxf(ps[6], 0.0f));
    const float excess = norm - radius;
    o.failed = false;  // the linear law has no damage
    if (!(excess > 0.0f)) {
        o.yielded = false;
        o.diss = 0.0f;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            o.sigma[i] = pressure + trial[i];
            o.sigma[3 + i] = trial[3 + i];
        }
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            o.n[i] = 0.0f;
            o.dp[i] = 0.0f;
        }
        o.theta = 1.0f;
        o.theta_bar = 0.0f;
        o.deq = 0.0f;
        return;
    }
    o.yielded = true;
    const float gamma = excess / (2.0f * p.mu + (2.0f / 3.0f) * p.hardening);
    const float inv_norm = 1.0f / norm;
#pragma unroll
    for (int i = 0; i < 6; ++i) o.n[i] = trial[i] * inv_norm;
    const float k = 2.0f * p.mu * gamma;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        o.sigma[i] = pressure + trial[i] - k * o.n[i];
        o.sigma[3 + i] = trial[3 + i] - k * o.n[3 + i];
        o.dp[i] = gamma * o.n[i];
        o.dp[3 + i] = 2.0f * gamma * o.n[3 + i];
    }
    o.deq = root23 * gamma;
    o.theta = 1.0f - k * inv_norm;
    o.theta_bar = 1.0f / (1.0f + p.hardening / (3.0f * p.mu)) - (1.0f - o.theta);
    float diss = 0.0f;
#pragma unroll
    for (int i = 0; i < 6; ++i) diss += o.sigma[i] * o.dp[i];
    o.diss = diss;
}

// Flow stress and its slope (plasticity.cpp:116-133): linear or Swift.
__device__ __forceinline__ float flow_stress(const ShellParams& p, float eq) {
    const float q = fmaxf(eq, 0.0f);
    return p.swift ? p.swift_k * powf(p.swift_eps0 + q, p.swift_n) : p.yield + p.hardening * q;
}

__device__ __forceinline__ float flow_slope(const ShellParams& p, float eq) {
    const float q = fmaxf(eq, 0.0f);
    return p.swift ? p.swift_k * p.swift_n * powf(p.swift_eps0 + q, p.swift_n - 1.0f) : p.hardening;
}

// The general point law (plasticity.cpp:319-505) from the point's start state: radial
// return against the back stress with the bracketed Newton on the consistency
// condition (FP32 tolerances: a few ulps of the yield radius and of the multiplier),
// back stress, damage with the triaxiality factor (plasticity.cpp:171-174), failure.
__device__ __forceinline__ void point_law_general(const float eps[6], const float ps[7], const float back0[6],
                                                  float damage0, bool failed0, float fstrain, const ShellParams& p,
                                                  PointOut& o) {
    o.yielded = false;
    o.failed = failed0;
    o.damage = damage0;
    o.deq = 0.0f;
    o.diss = 0.0f;
    o.theta = 1.0f;
    o.theta_bar = 0.0f;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        o.back[i] = back0[i];
        o.n[i] = 0.0f;
        o.dp[i] = 0.0f;
    }
    if (failed0) {
#pragma unroll
        for (int i = 0; i < 6; ++i) o.sigma[i] = 0.0f;
        o.theta = 0.0f;
        return;
    }
    float el[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) el[i] = eps[i] - ps[i];
    const float vol = el[0] + el[1] + el[2];
    const float pressure = p.kappa * vol;
    float trial[6], rel[6];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        trial[i] = 2.0f * p.mu * (el[i] - vol * (1.0f / 3.0f));
        trial[3 + i] = p.mu * el[3 + i];
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) rel[i] = trial[i] - back0[i];
    const float rnorm = sqrtf(rel[0] * rel[0] + rel[1] * rel[1] + rel[2] * rel[2] +
                              2.0f * (rel[3] * rel[3] + rel[4] * rel[4] + rel[5] * rel[5]));
    const float root23 = 0.81649658092772603f;
    const float radius = root23 * flow_stress(p, ps[6]);
    const float excess = rnorm - radius;
    if (!(excess > 0.0f)) {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            o.sigma[i] = pressure + trial[i];
            o.sigma[3 + i] = trial[3 + i];
        }
        return;
    }
    const float linear_part = 2.0f * p.mu + (2.0f / 3.0f) * p.kinematic;
    float lo = 0.0f, hi = excess / linear_part, gamma = hi;
#pragma unroll 1
    for (int it = 0; it < 50; ++it) {
        const float acc = ps[6] + root23 * gamma;
        const float res = rnorm - linear_part * gamma - root23 * flow_stress(p, acc);
        if (res > 0.0f)
            lo = gamma;
        else
            hi = gamma;
        if (fabsf(res) <= 5e-7f * radius) break;
        const float slope = -linear_part - (2.0f / 3.0f) * flow_slope(p, acc);
        float next = gamma - res / slope;
        if (!(next > lo && next < hi)) next = 0.5f * (lo + hi);
        if (fabsf(next - gamma) <= 1e-7f * gamma) {
            gamma = next;
            break;
        }
        gamma = next;
    }
    o.yielded = true;
    const float inv_norm = 1.0f / rnorm;
#pragma unroll
    for (int i = 0; i < 6; ++i) o.n[i] = rel[i] * inv_norm;
    const float k = 2.0f * p.mu * gamma;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        o.dp[i] = gamma * o.n[i];
        o.dp[3 + i] = 2.0f * gamma * o.n[3 + i];
        o.sigma[i] = pressure + trial[i] - k * o.n[i];
        o.sigma[3 + i] = trial[3 + i] - k * o.n[3 + i];
    }
    float diss = 0.0f;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        o.back[i] = back0[i] + (2.0f / 3.0f) * p.kinematic * gamma * o.n[i];
        diss += (o.sigma[i] - o.back[i]) * o.dp[i];
    }
    o.diss = diss;
    o.deq = root23 * gamma;
    // damage: Rice-Tracey factor on the triaxiality sigma_m / sigma_vm
    const float mean = (o.sigma[0] + o.sigma[1] + o.sigma[2]) * (1.0f / 3.0f);
    const float d0 = o.sigma[0] - mean, d1 = o.sigma[1] - mean, d2 = o.sigma[2] - mean;
    const float vm = sqrtf(1.5f * (d0 * d0 + d1 * d1 + d2 * d2 +
                                   2.0f * (o.sigma[3] * o.sigma[3] + o.sigma[4] * o.sigma[4] + o.sigma[5] * o.sigma[5])));
    const float eta = vm > 0.0f ? mean / vm : 0.0f;
    const float critical = eta <= p.tri_cut ? INFINITY : fstrain * expf(-p.tri_sens * (eta - p.tri_ref));
    if (critical > 0.0f && isfinite(critical)) o.damage += o.deq / critical;
    if (o.damage >= 1.0f) {
        o.damage = 1.0f;
        o.failed = true;
#pragma unroll
        for (int i = 0; i < 6; ++i) o.sigma[i] = 0.0f;
        o.theta = 0.0f;
        o.theta_bar = 0.0f;
        return;
    }
    o.theta = 1.0f - k * inv_norm;
    const float pm = flow_slope(p, ps[6] + o.deq) + p.kinematic;
    o.theta_bar = 1.0f / (1.0f + pm / (3.0f * p.mu)) - (1.0f - o.theta);
}

// C g for the algorithmic tangent C = kappa 1(x)1 + 2 mu theta I_dev - 2 mu thetaBar n(x)n
// in the reference's Voigt convention (engineering strain in, tensor stress out).
__device__ __forceinline__ void tangent_apply(const PointOut& o, const ShellParams& p, const float g[6], float out[6]) {
    if (o.failed) {  // a failed point carries nothing
#pragma unroll
        for (int i = 0; i < 6; ++i) out[i] = 0.0f;
        return;
    }
    const float tr = g[0] + g[1] + g[2];
    const float ng = o.n[0] * g[0] + o.n[1] * g[1] + o.n[2] * g[2] + o.n[3] * g[3] + o.n[4] * g[4] + o.n[5] * g[5];
    const float a = 2.0f * p.mu * o.theta, b = 2.0f * p.mu * o.theta_bar * ng;
#pragma unroll
    for (int i = 0; i < 3; ++i) out[i] = p.kappa * tr + a * (g[i] - tr * (1.0f / 3.0f)) - b * o.n[i];
#pragma unroll
    for (int i = 3; i < 6; ++i) out[i] = 0.5f * a * g[i] - b * o.n[i];
}

// Blocks per SM the register budget is sized for, chosen per launch.  With the
// operators formed in the kernel the element pass is issue- and latency-bound.  A zone
// that fills the GPU wants warps to hide latency, more than it minds spills: on the
// 2 M-element panel 4 blocks (128 registers, 16 warps per SM, ~30 bytes of spill)
// take 2.49 ms per pass, 5 (96 registers, 20 warps, ~310 bytes of spill to L1)
// 2.34 ms, 6 (85 registers, ~650 bytes) 2.74 ms.  A zone that fits in one wave is
// bound by one warp's dependent chain, where every spill reload is latency: on the
// reference's 2,048-element probe zone 3 blocks (168 registers, no spill) take 18.2 us
// per step, 4 blocks 19.7 us, 5 blocks 24.0 us.
constexpr int kShellMinbWide = 5;
constexpr int kShellMinbNarrow = 3;
constexpr int kShellWarpsNarrow = kShellMinbNarrow * kShellBlock / 32;  // per SM

// GENERAL: the general point law and the element failure rules (ShellParams::general);
// otherwise the linear law, whose state is only the plastic strain.
// EAS64: how much of the enhanced-strain block runs in FP64 (ShellParams::eas64): 0
// none; 1 the 7x7 factor and its substitutions; 2 also K_aa and the residual summed in
// double; 3 also alpha, its correction and its stored state (d.alpha64).
template <bool KAHAN, bool GENERAL, int MINB, int EAS64 = 0>
__global__ void __launch_bounds__(kShellBlock, MINB) shell_forces(ShellDevice d, ShellParams p) {
    // an inertial punch has stopped: the run is over (every thread reads the same flag)
    if (d.halt && *d.halt) return;
    const int lane = threadIdx.x & 31;
    const int gp = lane & 7;
    const long long group_raw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long e_raw = group_raw * 4 + (lane >> 3);
    const bool valid = e_raw < d.elements;
    // Tail lanes (past the last element, or whole warps past the last group) shadow the
    // last element and group for their loads and write nothing.
    const long long e = valid ? e_raw : d.elements - 1;
    const long long group = group_raw < d.groups ? group_raw : d.groups - 1;
    {
        // This warp's plastic state into L2 now, with one bulk prefetch, and the small
        // per-element rows with a line each.  The loads of them come after a dependent
        // chain (node ids, node rows, the rotation) that the registers cannot run ahead
        // of; prefetched, they hit L2 instead of DRAM.
        const void* st = d.state + (size_t)group * kShellStateQ * 32;
        if (lane == 1)
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(st), "r"((unsigned)(kShellStateQ * 32 * 4))
                         : "memory");
        const long long e0 = group * 4;  // <= elements - 1
        if (lane == 2) asm volatile("prefetch.global.L2 [%0];" ::"l"(d.index + e0 * 8));
        if (lane == 3) asm volatile("prefetch.global.L2 [%0];" ::"l"(d.slot + e0 * 8));
        if (lane == 4) asm volatile("prefetch.global.L2 [%0];" ::"l"(d.alpha + e0 * 8));
        if (lane == 5) asm volatile("prefetch.global.L2 [%0];" ::"l"(d.elem + e0 * kShellElemQ));
        if (lane == 6) {
            const long long last = d.elements * kShellElemQ - 1, at = e0 * kShellElemQ + 8;
            asm volatile("prefetch.global.L2 [%0];" ::"l"(d.elem + (at < last ? at : last)));
        }
    }
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const long long s = d.counter[0];
        d.counter[1] = s;
        d.counter[0] = s + 1;
    }

    // ---- the element's corners: lane g reads node g alone ----
    // Each lane forms its own corner's rest difference to corner 0 and displacement
    // difference to corner 0 (and, for a bottom corner, its director), each difference
    // taken as before: rest positions in double, rounded once; the compensated
    // displacement as a double-float.  The corners are parked in shared memory, one copy
    // per element (`geo`), where the element's eight lanes read them back.  One node read
    // per lane instead of eight, and no corner arrays held in registers.
    __shared__ __align__(16) float geo_park[kShellBlock / 8][kShellGeo];
    float* geo = geo_park[threadIdx.x >> 3];
    float dXg[3], ddg[3];
    {
        const int c0l = lane & 24;  // the lane of the element's corner 0
        const size_t og = (size_t)d.index[e * 8 + gp] * 3;
        const double Xg = d.rest[og], Yg = d.rest[og + 1], Zg = d.rest[og + 2];
        const float ug = d.disp[og], vg = d.disp[og + 1], wg = d.disp[og + 2];
        const double X0 = __shfl_sync(0xffffffffu, Xg, c0l), Y0 = __shfl_sync(0xffffffffu, Yg, c0l),
                     Z0 = __shfl_sync(0xffffffffu, Zg, c0l);
        // this corner's top node (bottom corners 0-3 use it for their director)
        const int topl = c0l + ((gp + 4) & 7);
        const double Xt = __shfl_sync(0xffffffffu, Xg, topl), Yt = __shfl_sync(0xffffffffu, Yg, topl),
                     Zt = __shfl_sync(0xffffffffu, Zg, topl);
        const float u0 = __shfl_sync(0xffffffffu, ug, c0l), v0 = __shfl_sync(0xffffffffu, vg, c0l),
                    w0 = __shfl_sync(0xffffffffu, wg, c0l);
        dXg[0] = (float)(Xg - X0);
        dXg[1] = (float)(Yg - Y0);
        dXg[2] = (float)(Zg - Z0);
        ddg[0] = ug - u0;
        ddg[1] = vg - v0;
        ddg[2] = wg - w0;
        if (KAHAN) {
            // the compensated displacement u - c as a double-float: the differences above
            // are exact (neighbouring values within a factor of two), and the difference
            // of the compensations restores the low bits u alone has lost
            const float cg0 = d.disp_c[og], cg1 = d.disp_c[og + 1], cg2 = d.disp_c[og + 2];
            const float c0 = __shfl_sync(0xffffffffu, cg0, c0l), c1 = __shfl_sync(0xffffffffu, cg1, c0l),
                        c2 = __shfl_sync(0xffffffffu, cg2, c0l);
            if (gp != 0) {
                ddg[0] -= cg0 - c0;
                ddg[1] -= cg1 - c1;
                ddg[2] -= cg2 - c2;
            }
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            geo[kGeoX + gp * 3 + i] = dXg[i];
            geo[kGeoDd + gp * 3 + i] = ddg[i];
        }
        if (gp < 4) {
            geo[kGeoD + gp * 3] = (float)(Xt - Xg);
            geo[kGeoD + gp * 3 + 1] = (float)(Yt - Yg);
            geo[kGeoD + gp * 3 + 2] = (float)(Zt - Zg);
        }
        __syncwarp();
    }
    // ---- the element row: J0^-1 and the enhanced-mode scales (all zero: no valid forms) ----
    float j0[9], cm[7];
    {
        const float4* row = d.elem + e * kShellElemQ;
        const float4 r0 = __ldg(row), r1 = __ldg(row + 1), r2 = __ldg(row + 2), r3 = __ldg(row + 3);
        const float v[16] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w, r2.x, r2.y, r2.z, r2.w, r3.x, r3.y, r3.z, r3.w};
#pragma unroll
        for (int k = 0; k < 9; ++k) j0[k] = v[k];
#pragma unroll
        for (int k = 0; k < 7; ++k) cm[k] = v[9 + k];
    }
    bool formed = false;
#pragma unroll
    for (int k = 0; k < 9; ++k) formed = formed || j0[k] != 0.0f;
    // ---- rotation: H = (sum_a dN_a(0) (x) dd_a) J0^-1, R = I + Q ----
    float q[9];
    {
        const float sx[8] = {-1, 1, 1, -1, -1, 1, 1, -1}, sy[8] = {-1, -1, 1, 1, -1, -1, 1, 1},
                    sz[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
        float jd[9];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f;
#pragma unroll
            for (int a = 0; a < 8; ++a) {
                const float v = geo[kGeoDd + a * 3 + i];
                a0 += sx[a] * v;
                a1 += sy[a] * v;
                a2 += sz[a] * v;
            }
            jd[i * 3] = 0.125f * a0;
            jd[i * 3 + 1] = 0.125f * a1;
            jd[i * 3 + 2] = 0.125f * a2;
        }
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) q[i * 3 + j] = jd[i * 3] * j0[j] + jd[i * 3 + 1] * j0[3 + j] + jd[i * 3 + 2] * j0[6 + j];
        // Higham iteration to convergence in FP32 (the CPU runs it to 1e-16 in double,
        // solid_shell.cpp:473-487), at most six iterations.  The iteration converges
        // quadratically: X = R (I + E) goes to R (I + E^2 / 2), and a step moves Q by
        // about |E|, so after a step of size s the next would move it by about s^2 / 2.
        // Stop once that is within an FP32 ulp of |Q| (s^2 <= 2.4e-7 |Q|), or once a
        // step itself moved Q by no more than a few ulps (4.8e-7 |Q|).
#pragma unroll 1
        for (int it = 0; it < 6; ++it) {
            float ipq[9], m[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) ipq[k] = q[k];
            ipq[0] += 1.0f;
            ipq[4] += 1.0f;
            ipq[8] += 1.0f;
            inv3f(ipq, m);
            float mq[9];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) mq[i * 3 + j] = m[i * 3] * q[j] + m[i * 3 + 1] * q[3 + j] + m[i * 3 + 2] * q[6 + j];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) ipq[i * 3 + j] = 0.5f * (q[i * 3 + j] - mq[j * 3 + i]);
            float step = 0.0f, size = 0.0f;
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                step = fmaxf(step, fabsf(ipq[k] - q[k]));
                size = fmaxf(size, fabsf(ipq[k]));
                q[k] = ipq[k];
            }
            if (step <= 4.8e-7f * size || step * step <= 2.4e-7f * size) break;
        }
    }
    // ---- co-rotated relative displacement u'_a = Q^T dX_a + dd_a + Q^T dd_a, lane a's
    // corner formed by lane a and parked beside the others ----
    {
        const float sx = dXg[0] + ddg[0];
        const float ty = dXg[1] + ddg[1];
        const float wz = dXg[2] + ddg[2];
#pragma unroll
        for (int i = 0; i < 3; ++i)
            geo[kGeoU + gp * 3 + i] = ddg[i] + (q[0 * 3 + i] * sx + q[1 * 3 + i] * ty + q[2 * 3 + i] * wz);
        __syncwarp();
    }
    const float(*dX)[3] = reinterpret_cast<const float(*)[3]>(geo + kGeoX);
    const float(*D)[3] = reinterpret_cast<const float(*)[3]>(geo + kGeoD);
    const float* u = geo + kGeoU;

    // the rotation waits in shared memory through the Newton iterations (each lane its
    // own copy: no synchronisation), freeing nine registers there
    __shared__ float q_park[9][kShellBlock];
#pragma unroll
    for (int k = 0; k < 9; ++k) q_park[k][threadIdx.x] = q[k];
    // ---- the point's operators, formed from the rest geometry ----
    const ShellLanePoint P = shell_lane_point(gp);
    float gx[3], gy[3], Ainv[9], w;
    shell_frame(dX, D, P, formed, gx, gy, Ainv, w);
    float eps_u[6];
    shell_strain(dX, D, u, P, gx, gy, Ainv, eps_u);
    // G factored: column j = gc_j T0[:, k_j], k = (0, 1, 2, 2, 2, 3, 3)
    // T0 is the element's, the same in its eight lanes: one copy in the element's record
    // in shared memory rather than 24 registers in every lane through the Newton loop
    float gc[7];
    {
        float T0[24];
        shell_t0(j0, T0);
        float4* t4 = reinterpret_cast<float4*>(geo + kGeoT);
#pragma unroll
        for (int k = 0; k < 6; ++k) t4[k] = make_float4(T0[4 * k], T0[4 * k + 1], T0[4 * k + 2], T0[4 * k + 3]);
        __syncwarp();
    }
    const float* T = geo + kGeoT;
    shell_enhanced_scales(cm, w, P, gc);
    // element volume and the energy scale sigma_y V
    const float volume = sum8(w);
    const float scale = p.yield * volume;
    // the size of this point's enhanced operator, for the residual's rounding floor
    float gnorm = 0.0f;
#pragma unroll
    for (int j = 0; j < 7; ++j) gnorm += gc[j] * gc[j];
    gnorm = sqrtf(gnorm);

    // ---- start-of-step state ----
    const size_t sbase = (size_t)group * kShellStateQ * 32 + lane;
    float ps[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) ps[k] = d.state[sbase + (size_t)k * 32];
    float back0[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f}, damage0 = 0.0f, fstrain = INFINITY;
    bool failed0 = false;
    const size_t sbase2 = (size_t)group * kShellState2Q * 32 + lane;
    if (GENERAL) {
#pragma unroll
        for (int k = 0; k < 6; ++k) back0[k] = d.state2[sbase2 + (size_t)k * 32];
        damage0 = d.state2[sbase2 + (size_t)6 * 32];
        failed0 = d.state2[sbase2 + (size_t)7 * 32] != 0.0f;
        fstrain = d.fail_strain[e];
    }
    // An element with a failed point runs without enhanced modes (solid_shell.cpp:871-874).
    bool eas_on = true;
    if (GENERAL) eas_on = ((__ballot_sync(0xffffffffu, failed0) >> (lane & 24)) & 0xffu) == 0u;
    float alpha[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) alpha[k] = eas_on ? d.alpha[e * 8 + k] : 0.0f;
    double alpha64[7];
    if constexpr (EAS64 >= 3) {
#pragma unroll
        for (int k = 0; k < 7; ++k) alpha64[k] = eas_on ? d.alpha64[e * 8 + k] : 0.0;
    }
    // the elastic K_aa factor of this element is usable (formed, and positive definite);
    // the FP64 variants form and factor K_aa every time
    const bool have_factor = EAS64 == 0 && d.kaa_factor != nullptr && __ldg(d.kaa_factor + e * 32) > 0.0f;

    // ---- EAS Newton ----
    // The four elements of a warp iterate together (the shuffles need the whole warp):
    // an element that has finished keeps re-evaluating at its final alpha, which
    // reproduces its final point state exactly, and applies no further correction.
    PointOut o;
    bool converged = false, done = false;
#pragma unroll 1
    for (int iteration = 0;; ++iteration) {
        // a finished element keeps its point state: the one at its final alpha
        if (!done) {
            float eps[6];
            if constexpr (EAS64 >= 3)
                shell_enhanced_apply64(T, gc, alpha64, eps_u, eps);
            else
                shell_enhanced_apply(T, gc, alpha, eps_u, eps);
            if (GENERAL)
                point_law_general(eps, ps, back0, damage0, failed0, fstrain, p, o);
            else
                point_law(eps, ps, p, o);
        }
        // r_j = sum_g w gc_j (T0[:, k_j] . sigma)
        float r[7];
        {
            float tau[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                float s = 0.0f;
#pragma unroll
                for (int i = 0; i < 6; ++i) s += T[k * 6 + i] * o.sigma[i];
                tau[k] = w * s;
            }
            const int kj[7] = {0, 1, 2, 2, 2, 3, 3};
#pragma unroll
            for (int j = 0; j < 7; ++j) r[j] = sum8(gc[j] * tau[kj[j]]);
        }
        double r64[7];
        if constexpr (EAS64 >= 2) {  // the residual summed in double
            double tau[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                double s = 0.0;
#pragma unroll
                for (int i = 0; i < 6; ++i) s += (double)T[k * 6 + i] * (double)o.sigma[i];
                tau[k] = (double)w * s;
            }
            const int kj[7] = {0, 1, 2, 2, 2, 3, 3};
#pragma unroll
            for (int j = 0; j < 7; ++j) r64[j] = sum8d((double)gc[j] * tau[kj[j]]);
        } else if constexpr (EAS64 == 1) {
#pragma unroll
            for (int j = 0; j < 7; ++j) r64[j] = (double)r[j];
        }
        // The rounding floor of the residual in FP32: a few ulps of the magnitude of its
        // terms, sum_g w |sigma_g| |gc_g| (T0's columns are unit vectors).  A residual
        // there is as converged as single precision allows; the tolerances below are
        // the reference's, scaled by sigma_y V, and reach far below it at low stress.
        float rfloor;
        {
            float sn = 0.0f;
#pragma unroll
            for (int i = 0; i < 6; ++i) sn += o.sigma[i] * o.sigma[i];
            rfloor = kResidualFloor * sum8(w * sqrtf(sn) * gnorm);
        }
        if (!done && !eas_on) {  // no enhanced modes: one evaluation is the update
            converged = true;
            done = true;
        }
        if (!done) {
            float rn = 0.0f;
#pragma unroll
            for (int k = 0; k < 7; ++k) rn += r[k] * r[k];
            if constexpr (EAS64 >= 2) {
                double rn64 = 0.0;
#pragma unroll
                for (int k = 0; k < 7; ++k) rn64 += r64[k] * r64[k];
                rn = (float)rn64;
            }
            if (sqrtf(rn) <= fmaxf(p.tol_residual * scale, rfloor)) {
                converged = true;
                done = true;
            } else if (iteration + 1 >= p.max_iterations) {
                done = true;
            }
        }
        if (__all_sync(0xffffffffu, done)) break;
        if constexpr (EAS64 == 0) {
        // An element whose eight points are all elastic at this iterate has the
        // elastic K_aa, whose Cholesky factor is formed once per material
        // (shell_elastic_factor).  The warp builds K_aa itself only when one of its
        // elements has a yielded point; the shuffles need the whole warp.
        const unsigned yielded_mask = __ballot_sync(0xffffffffu, o.yielded);
        const bool elastic_element = have_factor && ((yielded_mask >> (lane & 24)) & 0xffu) == 0u;
        if constexpr (EAS64 == 0) {
            // The work gate without the solve: |delta . r| = r^T K^-1 r <= trace(K^-1) |r|^2
            // for the elastic K_aa, so where the bound is under the gate the correction
            // would be turned down (as solid_shell.cpp:983-988 turns it down) and need not
            // be formed.  The element's factor is then not even read.
            if (!done && elastic_element) {
                float rn = 0.0f;
#pragma unroll
                for (int k = 0; k < 7; ++k) rn += r[k] * r[k];
                if (__ldg(d.kaa_factor + e * 32 + 28) * rn <= p.tol_work * scale) {
                    converged = true;
                    done = true;
                }
            }
            if (__all_sync(0xffffffffu, done)) break;
        }
        float l[28];
        bool spd = true;
        if (__any_sync(0xffffffffu, !elastic_element)) {
        // K_aa = sum_g w_g G^T C G, lower triangle: with G factored, the point's part is
        // gc_a gc_b H[k_a][k_b], H = T0c^T C T0c over T0's four columns (four tangent
        // applications rather than seven)
        float kaa[28];
        {
            float H[10];
#pragma unroll
            for (int kb = 0; kb < 4; ++kb) {
                float cg[6];
                tangent_apply(o, p, &T[kb * 6], cg);
#pragma unroll
                for (int ka = kb; ka < 4; ++ka) {
                    float s = 0.0f;
#pragma unroll
                    for (int i = 0; i < 6; ++i) s += T[ka * 6 + i] * cg[i];
                    H[ka * (ka + 1) / 2 + kb] = w * s;
                }
            }
            const int kj[7] = {0, 1, 2, 2, 2, 3, 3};
#pragma unroll
            for (int b = 0; b < 7; ++b)
#pragma unroll
                for (int a = b; a < 7; ++a)
                    kaa[a * (a + 1) / 2 + b] = sum8(gc[a] * gc[b] * H[kj[a] * (kj[a] + 1) / 2 + kj[b]]);
        }
        // Cholesky (solid_shell.cpp:432-457), identical in every lane
        {
            int t = 0;
#pragma unroll
            for (int i = 0; i < 7; ++i) {
#pragma unroll
                for (int j = 0; j <= i; ++j) {
                    float s = kaa[t];
#pragma unroll
                    for (int k = 0; k < j; ++k) s -= l[i * (i + 1) / 2 + k] * l[j * (j + 1) / 2 + k];
                    if (i == j) {  // the diagonal is kept as its reciprocal
                        spd = spd && (s > 0.0f);
                        l[t] = 1.0f / sqrtf(fmaxf(s, 1e-30f));
                    } else {
                        l[t] = s * l[j * (j + 1) / 2 + j];
                    }
                    ++t;
                }
            }
        }
        }
        if (elastic_element && !done) {
            const float4* lf = reinterpret_cast<const float4*>(d.kaa_factor + e * 32);
#pragma unroll
            for (int k = 0; k < 7; ++k) {
                const float4 v = __ldg(lf + k);
                l[4 * k] = v.x;
                l[4 * k + 1] = v.y;
                l[4 * k + 2] = v.z;
                l[4 * k + 3] = v.w;
            }
            spd = true;
        }
        // L L^T delta = -r; the factor's diagonal holds 1 / l_ii
        float delta[7];
#pragma unroll
        for (int i = 0; i < 7; ++i) {
            float s = -r[i];
#pragma unroll
            for (int k = 0; k < i; ++k) s -= l[i * (i + 1) / 2 + k] * delta[k];
            delta[i] = s * l[i * (i + 1) / 2 + i];
        }
#pragma unroll
        for (int i = 6; i >= 0; --i) {
            float s = delta[i];
#pragma unroll
            for (int k = i + 1; k < 7; ++k) s -= l[k * (k + 1) / 2 + i] * delta[k];
            delta[i] = s * l[i * (i + 1) / 2 + i];
        }
        float work = 0.0f;
#pragma unroll
        for (int k = 0; k < 7; ++k) work += delta[k] * r[k];
        // An element whose eight points are elastic, corrected with the exact elastic
        // factor, has its residual at zero to rounding after the correction: its stress
        // is linear in alpha, so the point state at the new alpha is the old one plus
        // C G delta, with no second evaluation, unless that stress would yield at a point
        // (then the iteration goes on as usual).  Linear law only.
        bool linear_try = false, linear_elastic = false;
        float sn[6];
        if (!done) {
            if (!spd) {
                done = true;  // no stiffness left in the enhanced modes: report, do not iterate
            } else if (fabsf(work) <= p.tol_work * scale) {
                converged = true;  // stop before applying, as solid_shell.cpp:983-988
                done = true;
            } else {
#pragma unroll
                for (int k = 0; k < 7; ++k) alpha[k] += delta[k];
                if (!GENERAL && elastic_element) {
                    const float zero[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
                    float de[6];
                    shell_enhanced_apply(T, gc, delta, zero, de);
                    const float dv = de[0] + de[1] + de[2];
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        sn[i] = o.sigma[i] + (p.kappa * dv + 2.0f * p.mu * (de[i] - dv * (1.0f / 3.0f)));
                        sn[3 + i] = o.sigma[3 + i] + p.mu * de[3 + i];
                    }
                    const float pr = (sn[0] + sn[1] + sn[2]) * (1.0f / 3.0f);
                    const float s0 = sn[0] - pr, s1 = sn[1] - pr, s2 = sn[2] - pr;
                    const float norm =
                        sqrtf(s0 * s0 + s1 * s1 + s2 * s2 + 2.0f * (sn[3] * sn[3] + sn[4] * sn[4] + sn[5] * sn[5]));
                    const float radius = 0.81649658092772603f * (p.yield + p.hardening * fmaxf(ps[6], 0.0f));
                    linear_try = true;
                    linear_elastic = norm <= radius;
                }
            }
        }
        if (!GENERAL) {
            // every lane takes part in the ballot; the decision is the element's
            const unsigned elastic_mask = __ballot_sync(0xffffffffu, linear_try && linear_elastic);
            if (linear_try && ((elastic_mask >> (lane & 24)) & 0xffu) == 0xffu) {
#pragma unroll
                for (int i = 0; i < 6; ++i) o.sigma[i] = sn[i];
                converged = true;
                done = true;
            }
        }
        } else {
            // The enhanced block with FP64 in it: K_aa (from the FP32 tangent, summed in
            // double from EAS64 = 2), its factor and the correction in double.
            double kaa64[28];
            {
                const int kj[7] = {0, 1, 2, 2, 2, 3, 3};
                if constexpr (EAS64 >= 2) {
                    double H[10];
#pragma unroll
                    for (int kb = 0; kb < 4; ++kb) {
                        float cg[6];
                        tangent_apply(o, p, &T[kb * 6], cg);
#pragma unroll
                        for (int ka = kb; ka < 4; ++ka) {
                            double s = 0.0;
#pragma unroll
                            for (int i = 0; i < 6; ++i) s += (double)T[ka * 6 + i] * (double)cg[i];
                            H[ka * (ka + 1) / 2 + kb] = (double)w * s;
                        }
                    }
#pragma unroll
                    for (int b = 0; b < 7; ++b)
#pragma unroll
                        for (int a = b; a < 7; ++a)
                            kaa64[a * (a + 1) / 2 + b] =
                                sum8d((double)gc[a] * (double)gc[b] * H[kj[a] * (kj[a] + 1) / 2 + kj[b]]);
                } else {
                    float H[10];
#pragma unroll
                    for (int kb = 0; kb < 4; ++kb) {
                        float cg[6];
                        tangent_apply(o, p, &T[kb * 6], cg);
#pragma unroll
                        for (int ka = kb; ka < 4; ++ka) {
                            float s = 0.0f;
#pragma unroll
                            for (int i = 0; i < 6; ++i) s += T[ka * 6 + i] * cg[i];
                            H[ka * (ka + 1) / 2 + kb] = w * s;
                        }
                    }
#pragma unroll
                    for (int b = 0; b < 7; ++b)
#pragma unroll
                        for (int a = b; a < 7; ++a)
                            kaa64[a * (a + 1) / 2 + b] =
                                (double)sum8(gc[a] * gc[b] * H[kj[a] * (kj[a] + 1) / 2 + kj[b]]);
                }
            }
            // Cholesky (solid_shell.cpp:432-457) in double, the diagonal kept as its reciprocal
            double l64[28];
            bool spd = true;
            {
                int t = 0;
#pragma unroll
                for (int i = 0; i < 7; ++i) {
#pragma unroll
                    for (int j = 0; j <= i; ++j) {
                        double s = kaa64[t];
#pragma unroll
                        for (int k = 0; k < j; ++k) s -= l64[i * (i + 1) / 2 + k] * l64[j * (j + 1) / 2 + k];
                        if (i == j) {
                            spd = spd && (s > 0.0);
                            l64[t] = 1.0 / sqrt(fmax(s, 1e-300));
                        } else {
                            l64[t] = s * l64[j * (j + 1) / 2 + j];
                        }
                        ++t;
                    }
                }
            }
            double delta64[7];
#pragma unroll
            for (int i = 0; i < 7; ++i) {
                double s = -r64[i];
#pragma unroll
                for (int k = 0; k < i; ++k) s -= l64[i * (i + 1) / 2 + k] * delta64[k];
                delta64[i] = s * l64[i * (i + 1) / 2 + i];
            }
#pragma unroll
            for (int i = 6; i >= 0; --i) {
                double s = delta64[i];
#pragma unroll
                for (int k = i + 1; k < 7; ++k) s -= l64[k * (k + 1) / 2 + i] * delta64[k];
                delta64[i] = s * l64[i * (i + 1) / 2 + i];
            }
            double work = 0.0;
#pragma unroll
            for (int k = 0; k < 7; ++k) work += delta64[k] * r64[k];
            if (!done) {
                if (!spd) {
                    done = true;
                } else if (fabs(work) <= (double)p.tol_work * (double)scale) {
                    converged = true;  // stop before applying, as solid_shell.cpp:983-988
                    done = true;
                } else if constexpr (EAS64 >= 3) {
#pragma unroll
                    for (int k = 0; k < 7; ++k) alpha64[k] += delta64[k];
                } else {
#pragma unroll
                    for (int k = 0; k < 7; ++k) alpha[k] += (float)delta64[k];
                }
            }
        }

    }

    // A point that failed in this step's Newton sends its element round once more
    // without enhanced modes, from the step's start state (solid_shell.cpp:990-996).  The
    // other elements of the warp re-evaluate at their final alpha, which reproduces
    // their points exactly.
    if (GENERAL) {
        // every lane takes part in the ballot (a short-circuit would leave lanes out of it)
        const unsigned failed_mask = __ballot_sync(0xffffffffu, o.failed);
        const bool died = eas_on && ((failed_mask >> (lane & 24)) & 0xffu) != 0u;
        if (__any_sync(0xffffffffu, died)) {
            if (died) {
                eas_on = false;
                converged = true;
#pragma unroll
                for (int k = 0; k < 7; ++k) alpha[k] = 0.0f;
                if constexpr (EAS64 >= 3) {
#pragma unroll
                    for (int k = 0; k < 7; ++k) alpha64[k] = 0.0;
                }
            }
            float eps[6];
            if constexpr (EAS64 >= 3)
                shell_enhanced_apply64(T, gc, alpha64, eps_u, eps);
            else
                shell_enhanced_apply(T, gc, alpha, eps_u, eps);
            point_law_general(eps, ps, back0, damage0, failed0, fstrain, p, o);
        }
    }

    // ---- commit ----
    double diss = 0.0, energy = 0.0;
    bool torn = false;
    if (GENERAL) torn = ((__ballot_sync(0xffffffffu, o.failed) >> (lane & 24)) & 0xffu) == 0xffu;
    if (GENERAL && valid && gp == 7) d.alpha[e * 8 + 7] = torn ? 1.0f : 0.0f;  // all eight points failed
    if (valid) {
        if (o.yielded) {
            diss = (double)w * (double)o.diss;
            if (KAHAN) {
                // the compensations are read only here, where a yielded point needs them
                float pc[7];
#pragma unroll
                for (int k = 0; k < 7; ++k) pc[k] = d.state[sbase + (size_t)(7 + k) * 32];
#pragma unroll
                for (int i = 0; i < 6; ++i) kahan_add(ps[i], pc[i], o.dp[i]);
                kahan_add(ps[6], pc[6], o.deq);
#pragma unroll
                for (int k = 0; k < 7; ++k) d.state[sbase + (size_t)(7 + k) * 32] = pc[k];
            } else {
#pragma unroll
                for (int i = 0; i < 6; ++i) ps[i] += o.dp[i];
                ps[6] += o.deq;
            }
#pragma unroll
            for (int k = 0; k < 7; ++k) d.state[sbase + (size_t)k * 32] = ps[k];
            if (GENERAL) {
#pragma unroll
                for (int k = 0; k < 6; ++k) d.state2[sbase2 + (size_t)k * 32] = o.back[k];
                d.state2[sbase2 + (size_t)6 * 32] = o.damage;
                d.state2[sbase2 + (size_t)7 * 32] = o.failed ? 1.0f : 0.0f;
            }
        }
        if constexpr (EAS64 >= 3) {
            // alpha in double; its FP32 copy is what the rest of the solver reads
#pragma unroll
            for (int k = 0; k < 7; ++k) alpha[k] = (float)alpha64[k];
            if (gp < 7) d.alpha64[e * 8 + gp] = alpha64[gp];
        }
        if (gp < 7) d.alpha[e * 8 + gp] = alpha[gp];
        const double s0 = o.sigma[0], s1 = o.sigma[1], s2 = o.sigma[2], s3 = o.sigma[3], s4 = o.sigma[4],
                     s5 = o.sigma[5];
        // 1/2 sigma : C^-1 : sigma = 1/2 [s_dev : s_dev / (2 mu) + p tr(sigma) / (3 kappa)],
        // p = tr(sigma) / 3, the engineering shears counted twice
        const double tr = s0 + s1 + s2;
        const double pr = tr * (1.0 / 3.0);
        const double d0 = s0 - pr, d1 = s1 - pr, d2 = s2 - pr;
        const double dev = d0 * d0 + d1 * d1 + d2 * d2 + 2.0 * (s3 * s3 + s4 * s4 + s5 * s5);
        energy = (double)w * 0.5 * (dev * p.inv_2mu + pr * tr * p.inv_3kappa);
    }

    // ---- f = -R sum_g w_g B_g^T sigma_g, reduce-scattered so lane a holds node a ----
    // (the rest corners back from shared memory and the point's frame formed again:
    // cheaper than holding them in registers through the Newton iterations)
    float f[24];
#pragma unroll
    for (int j = 0; j < 24; ++j) f[j] = 0.0f;
    {
        float fx[3], fy[3], Af[9], wf;
        shell_frame(dX, D, P, formed, fx, fy, Af, wf);
        shell_force(dX, D, P, fx, fy, Af, wf, o.sigma, f);
    }
    // round 1 (xor 4): keep nodes 0-3 (bit 2 clear) or 4-7
    const bool hi4 = (gp & 4) != 0, hi2 = (gp & 2) != 0, hi1 = (gp & 1) != 0;
#pragma unroll
    for (int j = 0; j < 12; ++j) {
        const float keep = hi4 ? f[12 + j] : f[j];
        const float give = hi4 ? f[j] : f[12 + j];
        f[j] = keep + __shfl_xor_sync(0xffffffffu, give, 4);
    }
#pragma unroll
    for (int j = 0; j < 6; ++j) {
        const float keep = hi2 ? f[6 + j] : f[j];
        const float give = hi2 ? f[j] : f[6 + j];
        f[j] = keep + __shfl_xor_sync(0xffffffffu, give, 2);
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const float keep = hi1 ? f[3 + j] : f[j];
        const float give = hi1 ? f[j] : f[3 + j];
        f[j] = keep + __shfl_xor_sync(0xffffffffu, give, 1);
    }
    if (valid) {
        // lane gp now holds sum over points of node gp's internal force; apply -R
        float* out = d.slots + (size_t)d.slot[e * 8 + gp] * 3;
        float qr[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) qr[k] = q_park[k][threadIdx.x];
#pragma unroll
        for (int i = 0; i < 3; ++i) out[i] = -(f[i] + (qr[i * 3] * f[0] + qr[i * 3 + 1] * f[1] + qr[i * 3 + 2] * f[2]));
    }
    // per-warp partials in fixed shuffle order: no block barrier, so a warp whose
    // elements converge early does not wait for the slowest warp of its block
    const unsigned nonconv = __ballot_sync(0xffffffffu, valid && gp == 0 && !converged);
    const unsigned ypts = __ballot_sync(0xffffffffu, valid && o.yielded);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        diss += __shfl_xor_sync(0xffffffffu, diss, off);
        energy += __shfl_xor_sync(0xffffffffu, energy, off);
    }
    if (lane == 0) {
        d.e_diss[group_raw] += diss;
        d.e_strain[group_raw] = energy;
        d.e_stats[group_raw * 2] += __popc(nonconv);
        d.e_stats[group_raw * 2 + 1] = __popc(ypts);
    }
}

template <bool KAHAN>
__device__ __forceinline__ void shell_move(float* u, float* uc, float v, float dt) {
    const float du = v * dt;
    if (KAHAN) {
        float c = *uc;
        float s = *u;
        kahan_add(s, c, du);
        *u = s;
        *uc = c;
    } else {
        *u += du;
    }
}

template <bool KAHAN>
__global__ void __launch_bounds__(kShellNodeBlock) shell_nodes(ShellDevice d, ShellParams p) {
    __shared__ double scratch[32];
    if (d.halt && *d.halt) return;  // an inertial punch has stopped: the run is over
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double work = 0.0, kin = 0.0, pwork = 0.0, damp = 0.0, bwork = 0.0;
    if (n < d.nodes) {
        const double t = (double)(d.counter[1] + 1) * p.dt64;  // the time at the step's end
        const float lf = p.rise_time > 0.0 ? (float)(t / p.rise_time < 1.0 ? t / p.rise_time : 1.0) : 1.0f;
        float force[3] = {0.0f, 0.0f, 0.0f};
        const uint32_t b = d.offset[n], e = d.offset[n + 1];
        const float* sl = d.slots + (size_t)b * 3;
#pragma unroll 4
        for (uint32_t k = b; k < e; ++k, sl += 3) {
            force[0] += sl[0];
            force[1] += sl[1];
            force[2] += sl[2];
        }
        // the stiffeners' forces through their ties, after the plating, in fibre order
        if (d.fibers) {
            for (uint32_t k = d.fiber_offset[n]; k < d.fiber_offset[n + 1]; ++k) {
                const float* fs = d.fiber_slots + (size_t)d.fiber_entry[k] * 3;
                force[0] += fs[0];
                force[1] += fs[1];
                force[2] += fs[2];
            }
        }
        const uint8_t pin = d.pinned[n];
        const float im = d.inv_mass[n], m = d.mass[n];
        float* vel = d.velocity + (size_t)n * 3;
        float* u = d.disp + (size_t)n * 3;
        float* uc = d.disp_c + (size_t)n * 3;
        // force -> velocity; a driven edge DOF keeps the velocity it would have taken,
        // for its work (zone.cpp:1094-1111)
        float v3[3], ext[3], free_v[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            ext[k] = d.load ? lf * d.load[(size_t)n * 3 + k] : 0.0f;
            float v = vel[k];
            if (pin & (1u << k)) {
                if (pin & (8u << k)) free_v[k] = m > 0.0f ? v + (force[k] + ext[k]) * im * p.dt : v;
                v = 0.0f;
            } else if (m > 0.0f) {
                v += (force[k] + ext[k]) * im * p.dt;
            }
            v3[k] = v;
        }
        // the damping and the kinetic energy it removes (zone.cpp:1113-1121); the factor
        // is applied in double, as given (its float would be off by ~1e-8, which is 1e-5
        // of the loss 1 - d^2 at d = 0.999)
        if (p.damping64 != 1.0)
            damp = 0.5 * (double)m * ((double)v3[0] * v3[0] + (double)v3[1] * v3[1] + (double)v3[2] * v3[2]) *
                   (1.0 - p.damping64 * p.damping64);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float v = (float)((double)v3[k] * p.damping64);
            vel[k] = v;
            work += (double)ext[k] * (double)v * (double)p.dt;
        }
        // The driven edge, after the damping and before the punch (zone.cpp:1123-1145):
        // the velocity that lands the DOF on meshed + prescribed * smoothstep(t / ramp)
        // this step; the boundary's work is what that costs over the free velocity.
        if (pin & 0x38u) {
            const int row = d.edge_map[n];
            double fraction = 1.0;
            if (p.edge_ramp > 0.0) {
                const double r = fmin(1.0, fmax(0.0, t / p.edge_ramp));
                fraction = r * r * (3.0 - 2.0 * r);
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                if (!(pin & (8u << k))) continue;
                const double now = KAHAN ? (double)u[k] - (double)uc[k] : (double)u[k];
                const double target =
                    (d.edge_base[(size_t)row * 3 + k] + d.edge_drive[(size_t)row * 3 + k] * fraction - now) / p.dt64;
                bwork += (double)m * (target - (double)free_v[k]) * target;
                vel[k] = (float)target;
            }
        }
        // The prescribed punch holds the nodes it grips at -speed along its axis; the
        // impulse that takes is its work (zone.cpp:1190-1198; solidshell_integrate.comp).
        // After the edge, before the position update.  The inertial punch is the
        // one-block shell_punch kernel that follows: it moves the gripped nodes itself.
        bool gripped = d.driven && d.driven[n];
        if (gripped && !p.inertial) {
            const double t0 = (double)d.counter[1] * p.dt64;  // time at the start of the step
            const float speed = p.punch_ramp > 0.0 && t0 < p.punch_ramp ? (float)(p.punch_speed * (t0 / p.punch_ramp))
                                                                         : p.punch_speed;
            const float along = vel[0] * p.axis_x + vel[1] * p.axis_y + vel[2] * p.axis_z;
            const float change = -speed - along;
            vel[0] += change * p.axis_x;
            vel[1] += change * p.axis_y;
            vel[2] += change * p.axis_z;
            pwork = -((double)m * (double)change) * (double)speed;
            gripped = false;
        }
        if (!gripped) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float v = vel[k];
                shell_move<KAHAN>(u + k, uc + k, v, p.dt);
                kin += 0.5 * (double)m * (double)v * (double)v;
            }
        }
    }
    const double bw = block_sum(work, scratch);
    const double bk = block_sum(kin, scratch);
    const double bp = d.driven && !p.inertial ? block_sum(pwork, scratch) : 0.0;
    const double bd = p.damping64 != 1.0 ? block_sum(damp, scratch) : 0.0;
    const double be = d.edge_map ? block_sum(bwork, scratch) : 0.0;
    if (threadIdx.x == 0) {
        d.n_work[blockIdx.x] += bw;
        d.n_kin[blockIdx.x] = bk;
        if (d.driven && !p.inertial) d.n_punch[blockIdx.x] += bp;
        if (p.damping64 != 1.0) d.n_damp[blockIdx.x] += bd;
        if (d.edge_map) d.n_edge[blockIdx.x] += be;
    }
}

// flowStress / flowSlope of the fibres' curve (plasticity.cpp:124-142), in double
__device__ __forceinline__ double fiber_flow_stress(const ShellParams::FiberLaw& m, double eq) {
    const double q = fmax(0.0, eq);
    return m.swift ? m.swift_k * pow(m.swift_eps0 + q, m.swift_n) : m.yield + m.hardening * q;
}
__device__ __forceinline__ double fiber_flow_slope(const ShellParams::FiberLaw& m, double eq) {
    const double q = fmax(0.0, eq);
    return m.swift ? m.swift_k * m.swift_n * pow(m.swift_eps0 + q, m.swift_n - 1.0) : m.hardening;
}

// The fibre's uniaxial return (constraint.cpp:39-95): backward Euler on the flow rule
// with isotropic hardening, the consistency condition solved by Newton (at most 32
// iterations, 1e-13 relative), then the damage increment with the bar's closed-form
// triaxiality +-1/3 (constraint.cpp:102-109).  st: plastic strain, eq. plastic strain,
// damage, failed.
__device__ __forceinline__ double fiber_return(const ShellParams::FiberLaw& m, double failure_strain, double strain,
                                               double st[4], double& dissipation_per_volume) {
    dissipation_per_volume = 0.0;
    if (st[3] != 0.0) return 0.0;
    const double trial = m.youngs * (strain - st[0]);
    const double yield = fiber_flow_stress(m, st[1]);
    if (fabs(trial) <= yield) return trial;
    double increment = (fabs(trial) - yield) / (m.youngs + fiber_flow_slope(m, st[1]));
    for (int it = 0; it < 32; ++it) {
        const double residual = fabs(trial) - m.youngs * increment - fiber_flow_stress(m, st[1] + increment);
        if (fabs(residual) <= 1e-13 * (yield + fabs(trial))) break;
        const double slope = m.youngs + fiber_flow_slope(m, st[1] + increment);
        if (!(slope > 0.0)) break;
        increment += residual / slope;
        if (increment < 0.0) increment = 0.0;
    }
    const double direction = trial >= 0.0 ? 1.0 : -1.0;
    const double stress = trial - direction * m.youngs * increment;
    st[0] += direction * increment;
    st[1] += increment;
    dissipation_per_volume = fabs(stress) * increment;
    const double eta = stress == 0.0 ? 0.0 : (stress > 0.0 ? 1.0 : -1.0) / 3.0;
    const double factor = eta <= m.tri_cut ? INFINITY : exp(-m.tri_sens * (eta - m.tri_ref));
    const double critical = failure_strain * factor;
    if (critical > 0.0 && isfinite(critical)) st[2] += increment / critical;
    if (st[2] >= 1.0) {
        st[2] = 1.0;
        st[3] = 1.0;
        return 0.0;
    }
    return stress;
}

// Constraint fibres (constraint.cpp:198-258), one thread per fibre in FP64: the tied
// end points from the positions at the start of the step (rest + u - c), the
// co-rotational axial strain (l - L) / L, the uniaxial return, and N = sigma A along
// the current axis, split over each end's node pair by the tie weights.  Written to
// the fibre's four force slots; the node pass gathers them.
template <bool KAHAN>
__global__ void __launch_bounds__(kShellFiberBlock) shell_fibers(ShellDevice d, ShellParams p) {
    __shared__ double scratch[64];
    if (d.halt && *d.halt) return;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double diss = 0.0, energy = 0.0;
    if (i < d.fibers) {
        float out[4][3] = {{0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}};
        const double rest_length = d.fiber_length[i], area = d.fiber_area[i];
        if (rest_length > 0.0 && area > 0.0) {
            const uint4 t = d.fiber_tie[i];
            const double2 w = d.fiber_weight[i];
            const uint32_t node[4] = {t.x, t.y, t.z, t.w};
            const double weight[2] = {w.x, w.y};
            double pos[4][3];
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const size_t o = (size_t)node[j] * 3 + k;
                    const double u = KAHAN ? (double)d.disp[o] - (double)d.disp_c[o] : (double)d.disp[o];
                    pos[j][k] = d.rest[o] + u;
                }
            double span[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const double a = pos[0][k] * (1.0 - weight[0]) + pos[1][k] * weight[0];
                const double b = pos[2][k] * (1.0 - weight[1]) + pos[3][k] * weight[1];
                span[k] = b - a;
            }
            const double l = sqrt(span[0] * span[0] + span[1] * span[1] + span[2] * span[2]);
            if (l > 0.0) {
                double st[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) st[k] = d.fiber_state[i * 4 + k];
                double dpv = 0.0;
                const double stress = fiber_return(p.fiber, d.fiber_fail[i], (l - rest_length) / rest_length, st, dpv);
#pragma unroll
                for (int k = 0; k < 4; ++k) d.fiber_state[i * 4 + k] = st[k];
                diss = dpv * area * rest_length;
                const double axial = stress * area;
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const double sa = e == 0 ? axial : -axial;
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const double f = span[k] / l * sa;
                        out[2 * e][k] = (float)((1.0 - weight[e]) * f);
                        out[2 * e + 1][k] = (float)(weight[e] * f);
                    }
                }
                energy = 0.5 * stress * stress / p.fiber.youngs * area * rest_length;
            }
        }
        float* slot = d.fiber_slots + (size_t)i * 12;
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int k = 0; k < 3; ++k) slot[j * 3 + k] = out[j][k];
    }
    block_sum2(diss, energy, scratch);
    if (threadIdx.x == 0) {
        d.f_diss[blockIdx.x] += diss;
        d.f_energy[blockIdx.x] = energy;
    }
}

// The inertial punch (zone.cpp:1154-1198), one block after the node pass.  The grip is
// a perfectly inelastic collision of the striking body with the gripped nodes:
// momentum along the axis is conserved, V' = (M V + sum_i m_i u_i) / (M + sum_i m_i)
// with u_i each node's speed along -axis; then every gripped node moves at V' along
// -axis, the impulse that takes is the resisting force, and its work is the punch's.
// The sums run in a fixed order (strided per thread, then block_sum), so the run is
// deterministic.  A body that has stopped (V' <= 0) sets the halt flag, and every
// kernel of the following steps returns at once, as zone::Solver ends the run
// (zone.cpp:1225-1230).
template <bool KAHAN>
__global__ void __launch_bounds__(kShellPunchBlock) shell_punch(ShellDevice d, ShellParams p) {
    __shared__ double scratch[32];
    __shared__ double speed_s;
    if (*d.halt) return;
    double momentum = 0.0, gripped_mass = 0.0;
    for (int i = threadIdx.x; i < d.n_driven; i += blockDim.x) {
        const uint32_t n = d.driven_list[i];
        const float* v = d.velocity + (size_t)n * 3;
        const float along = v[0] * p.axis_x + v[1] * p.axis_y + v[2] * p.axis_z;
        const double m = d.mass[n];
        momentum -= m * (double)along;
        gripped_mass += m;
    }
    momentum = block_sum(momentum, scratch);
    gripped_mass = block_sum(gripped_mass, scratch);
    if (threadIdx.x == 0) {
        const double V = (p.punch_mass * d.punch_state[0] + momentum) / (p.punch_mass + gripped_mass);
        d.punch_state[0] = V;
        speed_s = V;
    }
    __syncthreads();
    const double V = speed_s;
    const float speed = (float)V;
    double impulse = 0.0, kin = 0.0;
    for (int i = threadIdx.x; i < d.n_driven; i += blockDim.x) {
        const uint32_t n = d.driven_list[i];
        float* v = d.velocity + (size_t)n * 3;
        const float m = d.mass[n];
        const float along = v[0] * p.axis_x + v[1] * p.axis_y + v[2] * p.axis_z;
        const float change = -speed - along;
        v[0] += change * p.axis_x;
        v[1] += change * p.axis_y;
        v[2] += change * p.axis_z;
        impulse += (double)m * (double)change;
        float* u = d.disp + (size_t)n * 3;
        float* uc = d.disp_c + (size_t)n * 3;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            shell_move<KAHAN>(u + k, uc + k, v[k], p.dt);
            kin += 0.5 * (double)m * (double)v[k] * (double)v[k];
        }
    }
    impulse = block_sum(impulse, scratch);
    kin = block_sum(kin, scratch);
    if (threadIdx.x == 0) {
        const double force = -impulse / p.dt64;
        d.punch_state[1] += force * V * p.dt64;
        d.punch_state[2] += V * p.dt64;
        d.punch_state[3] += p.dt64;
        d.punch_state[4] += 1.0;
        *d.punch_kin = kin;
        if (!(V > 0.0)) *d.halt = 1;
    }
}

// The elastic K_aa = sum_g w_g G_g^T C G_g of every element, from the FP32 G and
// weights the step forms (shell_geom.cuh), accumulated in double, and its Cholesky
// factor (packed lower triangle, 28 of 32 floats per element, each diagonal entry
// stored as its reciprocal, as the step's own factorisation keeps it).  A zero first
// entry marks an element whose elastic K_aa is not positive definite; the step then
// forms K_aa itself.
__global__ void shell_elastic_factor(ShellDevice d, double lambda, double mu, float* out) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= d.elements) return;
    float Xb[4][3], D[4][3], a0[9], cm[7];
    shell_rest_corners(d, e, Xb, D);
    {
        const float* row = reinterpret_cast<const float*>(d.elem + e * kShellElemQ);
        for (int k = 0; k < 9; ++k) a0[k] = row[k];
        for (int k = 0; k < 7; ++k) cm[k] = row[9 + k];
    }
    bool formed = false;
    for (int k = 0; k < 9; ++k) formed = formed || a0[k] != 0.0f;
    float T[24];
    shell_t0(a0, T);
    double kaa[7][7];
    for (int a = 0; a < 7; ++a)
        for (int b = 0; b < 7; ++b) kaa[a][b] = 0.0;
    for (int gp = 0; gp < 8; ++gp) {
        const ShellLanePoint P = shell_lane_point(gp);
        float gx[3], gy[3], A[9], wf, g[42];
        shell_frame(Xb, D, P, formed, gx, gy, A, wf);
        shell_enhanced(T, cm, wf, P, g);
        const double w = wf;
        for (int b = 0; b < 7; ++b) {
            double col[6], cg[6];
            for (int i = 0; i < 6; ++i) col[i] = g[i * 7 + b];
            const double tr = col[0] + col[1] + col[2];
            for (int i = 0; i < 3; ++i) cg[i] = lambda * tr + 2.0 * mu * col[i];
            for (int i = 3; i < 6; ++i) cg[i] = mu * col[i];
            for (int a = 0; a < 7; ++a) {
                double s = 0.0;
                for (int i = 0; i < 6; ++i) s += (double)g[i * 7 + a] * cg[i];
                kaa[a][b] += w * s;
            }
        }
    }
    float l[32];
    double ld[28];
    bool spd = true;
    int t = 0;
    for (int i = 0; i < 7; ++i)
        for (int j = 0; j <= i; ++j) {
            double s = kaa[i][j];
            for (int k = 0; k < j; ++k) s -= ld[i * (i + 1) / 2 + k] * ld[j * (j + 1) / 2 + k];
            if (i == j) {
                spd = spd && s > 0.0;
                ld[t] = sqrt(s > 0.0 ? s : 1e-300);
            } else {
                ld[t] = s / ld[j * (j + 1) / 2 + j];
            }
            ++t;
        }
    for (int k = 0; k < 28; ++k) l[k] = (float)ld[k];
    for (int i = 0; i < 7; ++i) l[i * (i + 1) / 2 + i] = (float)(1.0 / ld[i * (i + 1) / 2 + i]);  // as the step keeps it
    // trace(K^-1) = |L^-1|_F^2, a bound on |K^-1|: the step decides the work gate
    // |delta . r| = r^T K^-1 r <= trace(K^-1) |r|^2 from it without solving, where it can
    double inv[28], trace = 0.0;
    for (int j = 0; j < 7; ++j)
        for (int i = j; i < 7; ++i) {
            double v = i == j ? 1.0 : 0.0;
            for (int k = j; k < i; ++k) v -= ld[i * (i + 1) / 2 + k] * inv[k * (k + 1) / 2 + j];
            inv[i * (i + 1) / 2 + j] = v / ld[i * (i + 1) / 2 + i];
            trace += inv[i * (i + 1) / 2 + j] * inv[i * (i + 1) / 2 + j];
        }
    l[28] = spd ? (float)(trace * (1.0 + 1e-4)) : 0.0f;  // a little over, for the rounding
    l[29] = l[30] = l[31] = 0.0f;
    if (!spd) l[0] = 0.0f;
    float4* o = reinterpret_cast<float4*>(out + e * 32);
    for (int k = 0; k < 8; ++k) o[k] = make_float4(l[4 * k], l[4 * k + 1], l[4 * k + 2], l[4 * k + 3]);
}

}  // namespace

void launch_shell_elastic_factor(const ShellDevice& d, double youngs, double poisson, float* out,
                                 cudaStream_t stream) {
    const double lambda = youngs * poisson / ((1.0 + poisson) * (1.0 - 2.0 * poisson));
    const double mu = youngs / (2.0 * (1.0 + poisson));
    shell_elastic_factor<<<blocks_for(d.elements, 128), 128, 0, stream>>>(d, lambda, mu, out);
}

template <int MINB>
static void launch_forces(const ShellDevice& d, const ShellParams& p, int blocks, cudaStream_t stream) {
    // the FP64 enhanced-block variants: compensated state and the general law only (the
    // host checks), at the narrow register budget
    if (p.eas64 == 1) {
        shell_forces<true, true, kShellMinbNarrow, 1><<<blocks, kShellBlock, 0, stream>>>(d, p);
        return;
    }
    if (p.eas64 == 2) {
        shell_forces<true, true, kShellMinbNarrow, 2><<<blocks, kShellBlock, 0, stream>>>(d, p);
        return;
    }
    if (p.eas64 == 3) {
        shell_forces<true, true, kShellMinbNarrow, 3><<<blocks, kShellBlock, 0, stream>>>(d, p);
        return;
    }
    if (p.compensated) {
        if (p.general)
            shell_forces<true, true, MINB><<<blocks, kShellBlock, 0, stream>>>(d, p);
        else
            shell_forces<true, false, MINB><<<blocks, kShellBlock, 0, stream>>>(d, p);
    } else {
        if (p.general)
            shell_forces<false, true, MINB><<<blocks, kShellBlock, 0, stream>>>(d, p);
        else
            shell_forces<false, false, MINB><<<blocks, kShellBlock, 0, stream>>>(d, p);
    }
}

void launch_shell_step(const ShellDevice& d, const ShellParams& p, cudaStream_t stream, int parts) {
    const int eb = blocks_for(d.groups * 32, kShellBlock);
    const int nb = blocks_for(d.nodes, kShellNodeBlock);
    const int fb = blocks_for(d.fibers, kShellFiberBlock);
    if ((parts & 1) && d.fibers) {
        if (p.compensated)
            shell_fibers<true><<<fb, kShellFiberBlock, 0, stream>>>(d, p);
        else
            shell_fibers<false><<<fb, kShellFiberBlock, 0, stream>>>(d, p);
    }
    // one wave at the narrow budget: the latency-bound form; else the wide one
    const bool narrow = d.groups <= (long long)d.sms * kShellWarpsNarrow;
    if (parts & 1) {
        if (narrow)
            launch_forces<kShellMinbNarrow>(d, p, eb, stream);
        else
            launch_forces<kShellMinbWide>(d, p, eb, stream);
    }
    if (p.compensated) {
        if (parts & 2) shell_nodes<true><<<nb, kShellNodeBlock, 0, stream>>>(d, p);
        if ((parts & 2) && p.inertial) shell_punch<true><<<1, kShellPunchBlock, 0, stream>>>(d, p);
    } else {
        if (parts & 2) shell_nodes<false><<<nb, kShellNodeBlock, 0, stream>>>(d, p);
        if ((parts & 2) && p.inertial) shell_punch<false><<<1, kShellPunchBlock, 0, stream>>>(d, p);
    }
}

}  // namespace fs
