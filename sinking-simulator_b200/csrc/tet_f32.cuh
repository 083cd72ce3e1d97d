// tet_f32.cuh -- the FP32 J2 tet element and node updates, shared by the single-mesh
// step (tet_fast.cu) and the batched / served pool (pool.cu).
//
// Same element and node update as the FP64 step (fem.cpp's co-rotational tet,
// plasticity::update's radial return, fem.cpp's node loop with a ramped external load),
// re-formulated so that FP32 keeps the digits that matter:
//
//   * nodes carry the displacement u = x - X (rest X fixed), not the position, so a
//     step's increment v dt ~ 1e-7 m is added to a number of size |u| ~ 1e-3 m rather
//     than |x| ~ 1 m.  The compensated variant adds it with Kahan summation and keeps
//     the pair (u, c), true value u - c, as a double-float: the element forms a
//     neighbour difference as (u_b - u_a) - (c_b - c_a), where the first difference is
//     exact (the two are within a factor of two, Sterbenz) and the second restores the
//     low bits u alone has lost.  A strain of 1e-4 on a displacement of 1e-2 m keeps
//     its digits instead of losing eleven bits to the subtraction;
//   * the element works on the displacement gradient H = Du Dm^-1 and the rotation's
//     deviation from identity Q = R - I, never on F = I + H and R themselves, so the
//     strain R^T F - I = H + Q^T + Q^T H is formed from small terms with no
//     cancellation.  The Higham iteration R <- (R + R^-T)/2 is carried in Q:
//     Q <- (Q - (M Q)^T)/2 with M = (I + Q)^-1 (fem.cpp:62-69), for as many steps as
//     FP32 needs at the tet's stretch (two for elastic steel, up to the reference's
//     four);
//   * the plastic strain is accumulated with Kahan compensation in the compensated
//     variant.
//
// Every file that includes this one is compiled without FMA contraction
// (-fmad=false); the fused multiply-adds below are written out (__fmaf_rn).  The
// arithmetic is then the same in every kernel that inlines these functions -- the
// single-mesh step, the pool's launches and its persistent kernel -- so a mesh gets
// the same bits whichever of them steps it.
#pragma once

#include "common.cuh"

namespace fs {

__device__ __forceinline__ void kahan_add(float& sum, float& comp, float x) {
    const float y = x - comp;
    const float t = sum + y;
    comp = (t - sum) - y;
    sum = t;
}

// a * b with each entry an explicit FMA chain: (a_i0 b_0j + a_i1 b_1j) + a_i2 b_2j
__device__ __forceinline__ M3<float> mul_fma(const M3<float>& a, const M3<float>& b) {
    M3<float> r;
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int i = 0; i < 3; ++i) r(i, c) = __fmaf_rn(a(i, 2), b(2, c), __fmaf_rn(a(i, 1), b(1, c), a(i, 0) * b(0, c)));
    return r;
}

// (I + Q)^-1 by the adjugate with FMA cofactors, for the Higham step.  A singular
// matrix (|det| <= tiny) gives zero, as fem.cpp's inverse does.
__device__ __forceinline__ M3<float> inverse_fma(const M3<float>& a, float tiny) {
    const float c00 = __fmaf_rn(a(1, 1), a(2, 2), -(a(1, 2) * a(2, 1)));
    const float c01 = __fmaf_rn(a(1, 2), a(2, 0), -(a(1, 0) * a(2, 2)));
    const float c02 = __fmaf_rn(a(1, 0), a(2, 1), -(a(1, 1) * a(2, 0)));
    const float det = __fmaf_rn(a(0, 2), c02, __fmaf_rn(a(0, 1), c01, a(0, 0) * c00));
    const float id = fabsf(det) > tiny ? 1.0f / det : 0.0f;
    M3<float> r;
    r(0, 0) = c00 * id;
    r(1, 0) = c01 * id;
    r(2, 0) = c02 * id;
    r(0, 1) = __fmaf_rn(a(0, 2), a(2, 1), -(a(0, 1) * a(2, 2))) * id;
    r(1, 1) = __fmaf_rn(a(0, 0), a(2, 2), -(a(0, 2) * a(2, 0))) * id;
    r(2, 1) = __fmaf_rn(a(0, 1), a(2, 0), -(a(0, 0) * a(2, 1))) * id;
    r(0, 2) = __fmaf_rn(a(0, 1), a(1, 2), -(a(0, 2) * a(1, 1))) * id;
    r(1, 2) = __fmaf_rn(a(0, 2), a(1, 0), -(a(0, 0) * a(1, 2))) * id;
    r(2, 2) = __fmaf_rn(a(0, 0), a(1, 1), -(a(0, 1) * a(1, 0))) * id;
    return r;
}

// A global load that bypasses L1 when CG: needed where another SM wrote the data
// earlier in the same (persistent) launch.
template <bool CG>
__device__ __forceinline__ float ldg_coherent(const float* p) {
    if (CG) return __ldcg(p);
    return *p;
}

template <bool CG>
__device__ __forceinline__ float4 ldg_coherent4(const float4* p) {
    if (CG) return __ldcg(p);
    return *p;
}

struct TetElementRefs {
    const uint4* index;     // [stride] node ids
    const uint4* slot;      // [stride] node-major slot of each corner
    const float* rest_inv;  // [9][stride]
    const float* rest_vol;  // [stride]
    float* plastic;         // [7][stride]
    float* plastic_c;       // [7][stride] (compensated variant)
    const float4* disp;     // [N] (ux, uy, uz, 0)
    const float4* disp_c;   // [N] Kahan compensation (compensated variant)
    float4* slots;          // [4 * stride]: one (fx, fy, fz, 0) per corner
    long long stride;       // SoA stride (tets, or the pool's tet capacity)
};

struct J2f {
    float mu, kappa, yield, hardening;
    // for the strain-energy density: 1 / (2 mu), 1 / (3 kappa)
    float inv_2mu_f, inv_3kappa_f;
};

// The material record of the FP32 J2 tet from the FP64 constants.
__host__ __device__ inline J2f make_j2f(double mu, double kappa, double yield, double hardening) {
    return J2f{(float)mu, (float)kappa, (float)yield, (float)hardening, (float)(1.0 / (2.0 * mu)),
               (float)(1.0 / (3.0 * kappa))};
}

// L2 prefetch of the per-tet rows of tets [begin, end) -- one 128-byte line per thread
// of the block: index (16 B per tet), slot map (16 B), Dm^-1 (9 rows of 4 B), volume
// and the plastic state (7 rows).  A block issues it for the tile one wave ahead, so
// that block's first loads, the ones whose results the gathers wait for, hit L2.  Every
// address lies inside [begin, end) of its row.
__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

__device__ __forceinline__ void prefetch_tet_rows(const TetElementRefs& d, long long begin, long long end) {
    if (end <= begin) return;
    const int x = threadIdx.x;
    const long long n = end - begin;
    const int wide = (int)((n * 16 + 127) >> 7);   // lines of a 16-byte row
    const int narrow = (int)((n * 4 + 127) >> 7);  // lines of a 4-byte row
    // each 4-byte row gets a power-of-two count of threads (no integer division);
    // threads past the row's last line issue nothing
    const int span = narrow <= 1 ? 1 : 1 << (32 - __clz(narrow - 1));
    const int shift = 31 - __clz(span);
    int k = x;
    if (k < wide) {
        prefetch_l2(reinterpret_cast<const char*>(d.index + begin) + ((long long)k << 7));
        return;
    }
    k -= wide;
    if (k < wide) {
        prefetch_l2(reinterpret_cast<const char*>(d.slot + begin) + ((long long)k << 7));
        return;
    }
    k -= wide;
    const int row = k >> shift, line = k & (span - 1);
    if (line >= narrow) return;
    const float* base;
    if (row < 9)
        base = d.rest_inv + (size_t)row * d.stride;
    else if (row == 9)
        base = d.rest_vol;
    else if (row < 17)
        base = d.plastic + (size_t)(row - 10) * d.stride;
    else
        return;
    prefetch_l2(reinterpret_cast<const char*>(base + begin) + ((long long)line << 7));
}

// Where a tet's own rows (node ids, slot map, Dm^-1, volume, plastic state) are read:
// straight from global memory, or from a block's copy of its tile in shared memory.
struct GlobalRows {
    const TetElementRefs& d;
    __device__ __forceinline__ uint4 index(long long t) const { return d.index[t]; }
    __device__ __forceinline__ uint4 slot(long long t) const { return d.slot[t]; }
    __device__ __forceinline__ float inv(int k, long long t) const { return d.rest_inv[(size_t)k * d.stride + t]; }
    __device__ __forceinline__ float vol(long long t) const { return d.rest_vol[t]; }
    __device__ __forceinline__ float plastic(int i, long long t) const { return d.plastic[(size_t)i * d.stride + t]; }
};

// A tile's rows in shared memory: index and slot map per tet from `first`, and 17
// float rows (Dm^-1 0..8, volume 9, plastic state 10..16) of `pitch` floats each from
// `base` (`first` rounded down to a multiple of 4, the 16-byte boundary of a row).
struct SharedRows {
    const uint4* idx;
    const uint4* slt;
    const float* rows;
    int pitch;
    long long first, base;
    __device__ __forceinline__ uint4 index(long long t) const { return idx[t - first]; }
    __device__ __forceinline__ uint4 slot(long long t) const { return slt[t - first]; }
    __device__ __forceinline__ float inv(int k, long long t) const { return rows[k * pitch + (int)(t - base)]; }
    __device__ __forceinline__ float vol(long long t) const { return rows[9 * pitch + (int)(t - base)]; }
    __device__ __forceinline__ float plastic(int i, long long t) const {
        return rows[(10 + i) * pitch + (int)(t - base)];
    }
};

// One tet from its four corners' displacements un (and compensations cn), however
// they were fetched: its four corner forces into fc (x, y, z, 0), its plastic state
// advanced; the dissipation and strain energy of the element in diss / energy (FP64,
// for the energy account).  The arithmetic is the same whichever `Rows` supplies the
// tet's own rows.
template <bool KAHAN, class Rows>
__device__ __forceinline__ void tet_element_f32_eval(const TetElementRefs& d, const Rows& rows, long long t,
                                                     const J2f& m, const float4 (&un)[4], const float4 (&cn)[4],
                                                     double& diss, double& energy, float4 (&fc)[4]) {
    M3<float> du, dm_inv;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        du(0, c) = un[c + 1].x - un[0].x;
        du(1, c) = un[c + 1].y - un[0].y;
        du(2, c) = un[c + 1].z - un[0].z;
        if (KAHAN) {  // true value u - c
            du(0, c) -= cn[c + 1].x - cn[0].x;
            du(1, c) -= cn[c + 1].y - cn[0].y;
            du(2, c) -= cn[c + 1].z - cn[0].z;
        }
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) dm_inv.m[k] = rows.inv(k, t);
    const M3<float> h = mul_fma(du, dm_inv);  // displacement gradient
    // rotation deviation Q = R - I by the Higham iteration on F = I + H.  Each step
    // squares the stretch error and halves it (F = R (I + E) goes to R (I + E^2 / 2)),
    // starting from about |sym H|, so the steps to reach FP32's relative precision of
    // the strain itself are known before the first: two up to |sym H| = 8e-3, three up
    // to 0.1, the reference's four beyond (fem.cpp:62-69 always takes four).
    const float e0 = fmaxf(fmaxf(fmaxf(fabsf(h(0, 0)), fabsf(h(1, 1))), fmaxf(fabsf(h(2, 2)), fabsf(h(0, 1) + h(1, 0)))),
                           fmaxf(fabsf(h(1, 2) + h(2, 1)), fabsf(h(2, 0) + h(0, 2))));
    const int higham_steps = e0 <= 8e-3f ? 2 : (e0 <= 0.1f ? 3 : 4);
    M3<float> q = h;
#pragma unroll 1
    for (int it = 0; it < higham_steps; ++it) {
        M3<float> ipq = q;
        ipq(0, 0) += 1.0f;
        ipq(1, 1) += 1.0f;
        ipq(2, 2) += 1.0f;
        const M3<float> mq = mul_fma(inverse_fma(ipq, 1e-30f), q);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) ipq(i, j) = 0.5f * (q(i, j) - mq(j, i));
        q = ipq;
    }
    const M3<float> qt = transpose(q);
    const M3<float> qth = mul_fma(qt, h);
    float strain[6];
    strain[0] = h(0, 0) + qt(0, 0) + qth(0, 0);
    strain[1] = h(1, 1) + qt(1, 1) + qth(1, 1);
    strain[2] = h(2, 2) + qt(2, 2) + qth(2, 2);
    strain[3] = (h(0, 1) + qt(0, 1) + qth(0, 1)) + (h(1, 0) + qt(1, 0) + qth(1, 0));
    strain[4] = (h(1, 2) + qt(1, 2) + qth(1, 2)) + (h(2, 1) + qt(2, 1) + qth(2, 1));
    strain[5] = (h(2, 0) + qt(2, 0) + qth(2, 0)) + (h(0, 2) + qt(0, 2) + qth(0, 2));

    // radial return, linear isotropic hardening (plasticity.cpp:333-456); for a linear
    // curve the consistency condition is affine in dgamma and its root is the closed
    // form below, which the CPU's Newton reaches in one step.
    float ps[7];
#pragma unroll
    for (int i = 0; i < 7; ++i) ps[i] = rows.plastic(i, t);
    float el[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) el[i] = strain[i] - ps[i];
    const float vol_strain = el[0] + el[1] + el[2];
    const float pressure = m.kappa * vol_strain;
    float trial[6];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        trial[i] = 2.0f * m.mu * (el[i] - vol_strain * (1.0f / 3.0f));
        trial[3 + i] = m.mu * el[3 + i];
    }
    const float norm = sqrtf(trial[0] * trial[0] + trial[1] * trial[1] + trial[2] * trial[2] +
                             2.0f * (trial[3] * trial[3] + trial[4] * trial[4] + trial[5] * trial[5]));
    const float root23 = 0.81649658092772603f;
    const float radius = root23 * (m.yield + m.hardening * fmaxf(ps[6], 0.0f));
    const float excess = norm - radius;
    float sv[6];
    diss = 0.0;
    if (excess > 0.0f) {
        const float gamma = excess / (2.0f * m.mu + (2.0f / 3.0f) * m.hardening);
        const float inv_norm = 1.0f / norm;
        const float k = 2.0f * m.mu * gamma * inv_norm;
        float dp[6];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            dp[i] = gamma * (trial[i] * inv_norm);
            sv[i] = pressure + __fmaf_rn(-k, trial[i], trial[i]);
        }
#pragma unroll
        for (int i = 3; i < 6; ++i) {
            dp[i] = 2.0f * gamma * (trial[i] * inv_norm);
            sv[i] = __fmaf_rn(-k, trial[i], trial[i]);
        }
        float dsum = 0.0f;
#pragma unroll
        for (int i = 0; i < 6; ++i) dsum += sv[i] * dp[i];
        diss = (double)dsum;
        const float deq = root23 * gamma;
        if (KAHAN) {
            // the compensation is read only where the state changes
            float pc[7];
#pragma unroll
            for (int i = 0; i < 7; ++i) pc[i] = d.plastic_c[(size_t)i * d.stride + t];
#pragma unroll
            for (int i = 0; i < 6; ++i) kahan_add(ps[i], pc[i], dp[i]);
            kahan_add(ps[6], pc[6], deq);
#pragma unroll
            for (int i = 0; i < 7; ++i) d.plastic_c[(size_t)i * d.stride + t] = pc[i];
        } else {
#pragma unroll
            for (int i = 0; i < 6; ++i) ps[i] += dp[i];
            ps[6] += deq;
        }
#pragma unroll
        for (int i = 0; i < 7; ++i) d.plastic[(size_t)i * d.stride + t] = ps[i];
    } else {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            sv[i] = pressure + trial[i];
            sv[3 + i] = trial[3 + i];
        }
    }
    const float volf = rows.vol(t);
    diss *= (double)volf;
    {
        // 1/2 sigma : C^-1 : sigma = 1/2 [s_dev : s_dev / (2 mu) + p tr(sigma) / (3 kappa)]
        // with p = tr(sigma) / 3, the engineering shears counted twice; the density in
        // FP32 (a relative error of a few ulps per tet), the account summed in FP64
        const float tr = sv[0] + sv[1] + sv[2];
        const float pr = tr * (1.0f / 3.0f);
        const float d0 = sv[0] - pr, d1 = sv[1] - pr, d2 = sv[2] - pr;
        const float dev = d0 * d0 + d1 * d1 + d2 * d2 + 2.0f * (sv[3] * sv[3] + sv[4] * sv[4] + sv[5] * sv[5]);
        energy = (double)(volf * 0.5f * (dev * m.inv_2mu_f + pr * tr * m.inv_3kappa_f));
    }
    // P = R sigma = sigma + Q sigma; nodal forces f_c = -V (P Dm^-T) column c
    M3<float> sig;
    sig(0, 0) = sv[0];
    sig(1, 1) = sv[1];
    sig(2, 2) = sv[2];
    sig(0, 1) = sig(1, 0) = sv[3];
    sig(1, 2) = sig(2, 1) = sv[4];
    sig(2, 0) = sig(0, 2) = sv[5];
    const M3<float> qs = mul_fma(q, sig);
#pragma unroll
    for (int k = 0; k < 9; ++k) sig.m[k] += qs.m[k];
    const M3<float> hf = mul_fma(sig, transpose(dm_inv));
    const float scale = -volf;
    float f0[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float v[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            v[a] = scale * hf(a, c);
            f0[a] -= v[a];
        }
        fc[c + 1] = make_float4(v[0], v[1], v[2], 0.0f);
    }
    fc[0] = make_float4(f0[0], f0[1], f0[2], 0.0f);
}

// The same with the corner forces written to the node-major slots (one 16-byte store
// each).
template <bool KAHAN, class Rows>
__device__ __forceinline__ void tet_element_f32_corners(const TetElementRefs& d, const Rows& rows, long long t,
                                                        const J2f& m, const float4 (&un)[4], const float4 (&cn)[4],
                                                        double& diss, double& energy) {
    float4 fc[4];
    tet_element_f32_eval<KAHAN, Rows>(d, rows, t, m, un, cn, diss, energy, fc);
    const uint4 sl = rows.slot(t);
    d.slots[sl.y] = fc[1];
    d.slots[sl.z] = fc[2];
    d.slots[sl.w] = fc[3];
    d.slots[sl.x] = fc[0];
}

template <bool KAHAN, bool CG = false, class Rows = GlobalRows>
__device__ __forceinline__ void tet_element_f32(const TetElementRefs& d, const Rows& rows, long long t, const J2f& m,
                                                double& diss, double& energy) {
    const uint4 idx = rows.index(t);
    const unsigned nid[4] = {idx.x, idx.y, idx.z, idx.w};
    float4 un[4], cn[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) un[c] = ldg_coherent4<CG>(d.disp + nid[c]);
    if (KAHAN) {
#pragma unroll
        for (int c = 0; c < 4; ++c) cn[c] = ldg_coherent4<CG>(d.disp_c + nid[c]);
    }
    tet_element_f32_corners<KAHAN, Rows>(d, rows, t, m, un, cn, diss, energy);
}

template <bool KAHAN, bool CG = false>
__device__ __forceinline__ void tet_element_f32(const TetElementRefs& d, long long t, const J2f& m, double& diss,
                                                double& energy) {
    tet_element_f32<KAHAN, CG, GlobalRows>(d, GlobalRows{d}, t, m, diss, energy);
}

struct TetNodeRefs {
    const uint32_t* offset;  // CSR offsets (absolute slot positions)
    const float4* slots;
    const uint8_t* fixed;
    const float* mass;
    const float* inv_mass;
    const float* ext;        // may be null
    float* velocity;
    float4* disp;            // (ux, uy, uz, 0)
    float4* disp_c;          // compensated variant
};

// One node: CSR gather in order, external load, symplectic Euler on the displacement.
template <bool KAHAN, bool CG = false>
__device__ __forceinline__ void tet_node_f32(const TetNodeRefs& d, long long n, float lf, float dt, float gravity,
                                             float damping, double& work, double& kin, double& gwork) {
    work = kin = gwork = 0.0;
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
#pragma unroll 4
    for (uint32_t k = b; k < e; ++k) {
        const float4 f = ldg_coherent4<CG>(d.slots + k);
        force[0] += f.x;
        force[1] += f.y;
        force[2] += f.z;
    }
    float ext[3] = {0.0f, 0.0f, 0.0f};
    if (d.ext) {
#pragma unroll
        for (int k = 0; k < 3; ++k) ext[k] = lf * d.ext[(size_t)n * 3 + k];
    }
    const float im = d.inv_mass[n];
    float4 u4 = d.disp[n], c4 = KAHAN ? d.disp_c[n] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float* u = &u4.x;
    float* cu = &c4.x;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float v = vel[k] + (force[k] + ext[k]) * im * dt;
        v *= damping;
        vel[k] = v;
        const float du = v * dt;
        if (KAHAN)
            kahan_add(u[k], cu[k], du);
        else
            u[k] += du;
        work += (double)ext[k] * (double)v * (double)dt;
        kin += 0.5 * (double)m * (double)v * (double)v;
    }
    d.disp[n] = u4;
    if (KAHAN) d.disp_c[n] = c4;
    gwork = -(double)gravity * (double)m * (double)vel[2] * (double)dt;
}

}  // namespace fs
