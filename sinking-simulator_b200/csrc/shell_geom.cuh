// shell_geom.cuh -- the solid-shell element's strain-displacement and enhanced-strain
// operators, formed in FP32 inside the step from the rest geometry.
//
// The element is the reference's 8-node solid-shell with assumed transverse shear
// (Dvorkin-Bathe), assumed thickness strain (Betsch-Stein) and seven enhanced modes
// (engine/sim/solid_shell.cpp:60-375, computeForms).  Instead of streaming its B (6x24)
// and G (6x7) per Gauss point from memory, each lane forms the products it needs,
// eps = B u and f = B^T sigma w, from the rest corner positions:
//
//   corners c = 0..3 in the element plane (xi_c, eta_c) = (-1,-1), (1,-1), (1,1), (-1,1);
//   node c is corner c's bottom (zeta = -1), node c + 4 its top.  With
//   psi_c(xi, eta) = (1 + xi xi_c)(1 + eta eta_c) / 4, lo = (1 - zeta)/2, hi = (1 + zeta)/2:
//     X(xi, eta, zeta) = sum_c psi_c (X_c + hi D_c),   D_c = X_{c+4} - X_c (the director)
//     g_xi = sum_c psi_c,xi Xl_c,  g_eta = sum_c psi_c,eta Xl_c,  g_zeta = 1/2 sum_c psi_c D_c
//   where Xl_c = X_c + hi D_c is corner c at the point's own thickness level; the
//   displacement likewise (ul_c = lo u_c + hi u_{c+4}, V_c = u_{c+4} - u_c).
//
// Natural strains, Voigt [E11, E22, E33, 2E12, 2E23, 2E31] in (xi, eta, zeta)
// (naturalB, solid_shell.cpp:85-101):
//   E11 = g_xi . u,xi    E22 = g_eta . u,eta    2E12 = g_xi . u,eta + g_eta . u,xi
//   E33: the corners' g_zeta . u,zeta = D_c . V_c / 4, interpolated with psi_c
//        (sampleAns and the thickness cure, solid_shell.cpp:215-233, 300-309);
//   2E23: (1-xi)/2 S(0,3) + (1+xi)/2 S(1,2),  2E31: (1-eta)/2 S(0,1) + (1+eta)/2 S(3,2),
//        the edge-midpoint samples at the point's own zeta (solid_shell.cpp:290-299), with
//        S(m,p) = g_dir . u,zeta + g_zeta . u,dir at the midpoint of edge m -> p
//              = [(Xl_p - Xl_m) . (V_m + V_p) + (D_m + D_p) . (ul_p - ul_m)] / 8.
// Cartesian strain eps = A^T E A with A = J^-1 at the point (voigtTransform,
// solid_shell.cpp:113-143), J's columns the base vectors, so A's rows are the dual
// vectors g^k = (g_l x g_m) / det J.  The Gauss weight is det J (all 2x2x2 weights 1).
//
// The transpose: tau = T^T sigma is the natural stress S = A sigma A^T (conjugate to the
// engineering natural strains), and f_a = w sum_j tau_j dE_j / du_a term by term.
//
// Enhanced modes (enhancedM, solid_shell.cpp:169-179, and the Simo-Rifai scaling and
// normalisation of computeForms, :312-375): column j of G at a point is
//   G_j = (det J0 / det J) n_j m_j(xi, eta, zeta) T0[:, k_j],
// m = (xi, eta, zeta, xi zeta, eta zeta, xi, eta), k = (0, 1, 2, 2, 2, 3, 3), T0 the
// Voigt transform of J0^-1 (the centre), n_j the mode's rest-configuration norm.  The
// element row holds J0^-1 and c_j = det J0 n_j, formed once in FP64.
//
// Precision: the rest differences (X_c - X_0 and the directors D_c) are taken in double
// and rounded once, so a thin element's g_zeta keeps FP32's relative precision rather
// than losing the plate's aspect ratio to cancellation.
#pragma once

namespace fs {

struct ShellLanePoint {
    float xi, eta, zeta, lo, hi;
    float ps[4], px[4], py[4];  // psi_c and its xi, eta derivatives at (xi, eta)
};

__device__ __forceinline__ ShellLanePoint shell_lane_point(int gp) {
    const float q = 0.57735026918962576f;  // 1/sqrt(3)
    ShellLanePoint P;
    P.xi = (gp & 1) ? q : -q;
    P.eta = (gp & 2) ? q : -q;
    P.zeta = (gp & 4) ? q : -q;
    P.lo = 0.5f * (1.0f - P.zeta);
    P.hi = 0.5f * (1.0f + P.zeta);
    const float cx[4] = {-1.0f, 1.0f, 1.0f, -1.0f}, cy[4] = {-1.0f, -1.0f, 1.0f, 1.0f};
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const float ax = 1.0f + P.xi * cx[c], ay = 1.0f + P.eta * cy[c];
        P.ps[c] = 0.25f * ax * ay;
        P.px[c] = 0.25f * cx[c] * ay;
        P.py[c] = 0.25f * cy[c] * ax;
    }
    return P;
}

__device__ __forceinline__ float dot3(const float a[3], const float b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// Base vectors at the lane's point, the dual basis A (row k = g^k) and w = det J.
// ok false: A = 0, w = 0 (the element contributes nothing).
__device__ __forceinline__ void shell_frame(const float Xb[4][3], const float D[4][3], const ShellLanePoint& P, bool ok,
                                            float gx[3], float gy[3], float A[9], float& w) {
    float gz[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float sx = 0.0f, sy = 0.0f, sz = 0.0f;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const float xl = Xb[c][i] + P.hi * D[c][i];
            sx += P.px[c] * xl;
            sy += P.py[c] * xl;
            sz += P.ps[c] * D[c][i];
        }
        gx[i] = sx;
        gy[i] = sy;
        gz[i] = 0.5f * sz;
    }
    // g^0 = (g_eta x g_zeta) / det, g^1 = (g_zeta x g_xi) / det, g^2 = (g_xi x g_eta) / det
    const float c0[3] = {gy[1] * gz[2] - gy[2] * gz[1], gy[2] * gz[0] - gy[0] * gz[2], gy[0] * gz[1] - gy[1] * gz[0]};
    const float c1[3] = {gz[1] * gx[2] - gz[2] * gx[1], gz[2] * gx[0] - gz[0] * gx[2], gz[0] * gx[1] - gz[1] * gx[0]};
    const float c2[3] = {gx[1] * gy[2] - gx[2] * gy[1], gx[2] * gy[0] - gx[0] * gy[2], gx[0] * gy[1] - gx[1] * gy[0]};
    const float det = dot3(gx, c0);
    const float inv = ok && det != 0.0f ? 1.0f / det : 0.0f;
    w = ok ? det : 0.0f;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        A[i] = c0[i] * inv;
        A[3 + i] = c1[i] * inv;
        A[6 + i] = c2[i] * inv;
    }
}

// S(m, p) of the edge-midpoint assumed shear, as a function of the level corners.
__device__ __forceinline__ float shell_edge_sample(const float Xb[4][3], const float D[4][3], const float ul[4][3],
                                                   const float V[4][3], float hi, int m, int p) {
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float dxl = (Xb[p][i] + hi * D[p][i]) - (Xb[m][i] + hi * D[m][i]);
        s += dxl * (V[m][i] + V[p][i]) + (D[m][i] + D[p][i]) * (ul[p][i] - ul[m][i]);
    }
    return 0.125f * s;
}

// eps = B u at the lane's point; u = the 8 corners' co-rotated relative displacement.
__device__ __forceinline__ void shell_strain(const float Xb[4][3], const float D[4][3], const float u[24],
                                             const ShellLanePoint& P, const float gx[3], const float gy[3],
                                             const float A[9], float eps[6]) {
    float ul[4][3], V[4][3];
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            ul[c][i] = P.lo * u[c * 3 + i] + P.hi * u[(c + 4) * 3 + i];
            V[c][i] = u[(c + 4) * 3 + i] - u[c * 3 + i];
        }
    float ux[3], uy[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float sx = 0.0f, sy = 0.0f;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            sx += P.px[c] * ul[c][i];
            sy += P.py[c] * ul[c][i];
        }
        ux[i] = sx;
        uy[i] = sy;
    }
    float E[6];
    E[0] = dot3(gx, ux);
    E[1] = dot3(gy, uy);
    E[3] = dot3(gx, uy) + dot3(gy, ux);
    {
        float s = 0.0f;
#pragma unroll
        for (int c = 0; c < 4; ++c) s += P.ps[c] * dot3(D[c], V[c]);
        E[2] = 0.25f * s;
    }
    E[4] = 0.5f * (1.0f - P.xi) * shell_edge_sample(Xb, D, ul, V, P.hi, 0, 3) +
           0.5f * (1.0f + P.xi) * shell_edge_sample(Xb, D, ul, V, P.hi, 1, 2);
    E[5] = 0.5f * (1.0f - P.eta) * shell_edge_sample(Xb, D, ul, V, P.hi, 0, 1) +
           0.5f * (1.0f + P.eta) * shell_edge_sample(Xb, D, ul, V, P.hi, 3, 2);
    // eps = A^T Et A, Et the natural strain tensor (engineering shears halved)
    const float Et[9] = {E[0], 0.5f * E[3], 0.5f * E[5], 0.5f * E[3], E[1], 0.5f * E[4], 0.5f * E[5], 0.5f * E[4], E[2]};
    float W[9];  // W = Et A
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int c = 0; c < 3; ++c) W[k * 3 + c] = Et[k * 3] * A[c] + Et[k * 3 + 1] * A[3 + c] + Et[k * 3 + 2] * A[6 + c];
    float e[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = r; c < 3; ++c) e[r][c] = A[r] * W[c] + A[3 + r] * W[3 + c] + A[6 + r] * W[6 + c];
    eps[0] = e[0][0];
    eps[1] = e[1][1];
    eps[2] = e[2][2];
    eps[3] = 2.0f * e[0][1];
    eps[4] = 2.0f * e[1][2];
    eps[5] = 2.0f * e[0][2];
}

// f (8 corners x 3) += B^T (w sigma) at the lane's point.
__device__ __forceinline__ void shell_force(const float Xb[4][3], const float D[4][3], const ShellLanePoint& P,
                                            const float gx[3], const float gy[3], const float A[9], float w,
                                            const float sigma[6], float f[24]) {
    // natural stress S = A s A^T (s the stress tensor), times the weight
    const float s[9] = {sigma[0], sigma[3], sigma[5], sigma[3], sigma[1], sigma[4], sigma[5], sigma[4], sigma[2]};
    float Vm[9];  // Vm = s A^T: Vm[r][l] = sum_c s[r][c] A[l][c]
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int l = 0; l < 3; ++l) Vm[r * 3 + l] = s[r * 3] * A[l * 3] + s[r * 3 + 1] * A[l * 3 + 1] + s[r * 3 + 2] * A[l * 3 + 2];
    float S[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int l = k; l < 3; ++l) S[k][l] = w * (A[k * 3] * Vm[l] + A[k * 3 + 1] * Vm[3 + l] + A[k * 3 + 2] * Vm[6 + l]);
    const float t0 = S[0][0], t1 = S[1][1], t2 = S[2][2], t3 = S[0][1], t4 = S[1][2], t5 = S[0][2];
    // E11, E22, 2E12: corner c's level value carries lo to the bottom node, hi to the top
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float pv = t0 * gx[i] + t3 * gy[i];
        const float qv = t1 * gy[i] + t3 * gx[i];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const float F = P.px[c] * pv + P.py[c] * qv;
            f[c * 3 + i] += P.lo * F;
            f[(c + 4) * 3 + i] += P.hi * F;
        }
    }
    // E33 from the corners: d/dV_c = psi_c D_c / 4
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const float T = 0.25f * t2 * P.ps[c] * D[c][i];
            f[(c + 4) * 3 + i] += T;
            f[c * 3 + i] -= T;
        }
    // the four edge samples: dS/dV_m = dS/dV_p = (Xl_p - Xl_m) / 8, dS/dul_p = -dS/dul_m = (D_m + D_p) / 8
    const int em[4] = {0, 1, 0, 3}, ep[4] = {3, 2, 1, 2};
    const float kap[4] = {0.5f * (1.0f - P.xi) * t4, 0.5f * (1.0f + P.xi) * t4, 0.5f * (1.0f - P.eta) * t5,
                          0.5f * (1.0f + P.eta) * t5};
#pragma unroll
    for (int s4 = 0; s4 < 4; ++s4) {
        const int m = em[s4], p = ep[s4];
        const float k8 = 0.125f * kap[s4];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const float av = k8 * ((Xb[p][i] + P.hi * D[p][i]) - (Xb[m][i] + P.hi * D[m][i]));
            const float bv = k8 * (D[m][i] + D[p][i]);
            f[(m + 4) * 3 + i] += av - P.hi * bv;
            f[m * 3 + i] += -av - P.lo * bv;
            f[(p + 4) * 3 + i] += av + P.hi * bv;
            f[p * 3 + i] += -av + P.lo * bv;
        }
    }
}

// Columns 0-3 of T0, the Voigt transform of J0^-1 (row-major a0): 4 x 6, column-major.
__device__ __forceinline__ void shell_t0(const float a0[9], float T[24]) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float r0 = a0[k * 3], r1 = a0[k * 3 + 1], r2 = a0[k * 3 + 2];
        T[k * 6 + 0] = r0 * r0;
        T[k * 6 + 1] = r1 * r1;
        T[k * 6 + 2] = r2 * r2;
        T[k * 6 + 3] = 2.0f * r0 * r1;
        T[k * 6 + 4] = 2.0f * r1 * r2;
        T[k * 6 + 5] = 2.0f * r2 * r0;
    }
    T[18] = a0[0] * a0[3];
    T[19] = a0[1] * a0[4];
    T[20] = a0[2] * a0[5];
    T[21] = a0[0] * a0[4] + a0[1] * a0[3];
    T[22] = a0[1] * a0[5] + a0[2] * a0[4];
    T[23] = a0[2] * a0[3] + a0[0] * a0[5];
}

// G's per-point column scales gc_j = c_j m_j(xi, eta, zeta) / det J, so that G's column
// j is gc_j T0[:, k_j]; the step keeps G in this factored form (T0's four columns and
// seven scalars rather than 42 entries).
__device__ __forceinline__ void shell_enhanced_scales(const float c[7], float w, const ShellLanePoint& P, float gc[7]) {
    const float iw = w != 0.0f ? 1.0f / w : 0.0f;
    const float m[7] = {P.xi, P.eta, P.zeta, P.xi * P.zeta, P.eta * P.zeta, P.xi, P.eta};
#pragma unroll
    for (int j = 0; j < 7; ++j) gc[j] = c[j] * m[j] * iw;
}

// out = base + G alpha, G factored: T0 times the four combined mode coefficients.
__device__ __forceinline__ void shell_enhanced_apply(const float T[24], const float gc[7], const float alpha[7],
                                                     const float base[6], float out[6]) {
    const float b0 = gc[0] * alpha[0], b1 = gc[1] * alpha[1];
    const float b2 = gc[2] * alpha[2] + gc[3] * alpha[3] + gc[4] * alpha[4];
    const float b3 = gc[5] * alpha[5] + gc[6] * alpha[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) out[i] = base[i] + T[i] * b0 + T[6 + i] * b1 + T[12 + i] * b2 + T[18 + i] * b3;
}

// G (6 x 7, row-major) written out, for the elastic factor's set-up.
__device__ __forceinline__ void shell_enhanced(const float T[24], const float c[7], float w, const ShellLanePoint& P,
                                               float G[42]) {
    float gc[7];
    shell_enhanced_scales(c, w, P, gc);
    const int k[7] = {0, 1, 2, 2, 2, 3, 3};
#pragma unroll
    for (int j = 0; j < 7; ++j)
#pragma unroll
        for (int i = 0; i < 6; ++i) G[i * 7 + j] = gc[j] * T[k[j] * 6 + i];
}

}  // namespace fs
