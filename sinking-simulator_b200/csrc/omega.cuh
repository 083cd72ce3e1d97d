// omega.cuh -- the FP64 element frequency bound of a linear tet, for the critical step.
//
// (4 / rho) lambda_max(B^T C B) of the lumped-mass element by power iteration, as
// solidshell::criticalTimestep does for the hex (solid_shell.cpp:1088-1133): the
// Rayleigh quotient, at most 400 iterations, relative 1e-10, the same start vector.
// g holds the shape-function gradients of the four corners (Dm^-T rows, corner 0 the
// negative sum).  Included by files compiled without FMA contraction, so every caller
// gets the same bits.
#pragma once

namespace fs {

// SCALE_BY_RECIPROCAL: normalise the iterate by one reciprocal of its norm and twelve
// products instead of twelve divisions (a few times cheaper in FP64; the iterate differs
// by rounding, the converged bound by far less than the iteration's 1e-10).  The pool's
// admission uses it; the single-mesh bound keeps the divisions, bit-identical to the
// FP64 oracle's.
template <bool SCALE_BY_RECIPROCAL = false>
__device__ __forceinline__ double tet_omega2_one(const double g[4][3], double lambda, double mu, double rho) {
    double v[12];
#pragma unroll
    for (int i = 0; i < 12; ++i) v[i] = 1.0 + 0.37 * i - 0.11 * i * i;
    double lam = 0.0;
#pragma unroll 1
    for (int it = 0; it < 400; ++it) {
        double e[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            const double* u = &v[n * 3];
            e[0] += g[n][0] * u[0];
            e[1] += g[n][1] * u[1];
            e[2] += g[n][2] * u[2];
            e[3] += g[n][1] * u[0] + g[n][0] * u[1];
            e[4] += g[n][2] * u[1] + g[n][1] * u[2];
            e[5] += g[n][0] * u[2] + g[n][2] * u[0];
        }
        const double tr = e[0] + e[1] + e[2];
        double s[6];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            s[i] = lambda * tr + 2.0 * mu * e[i];
            s[3 + i] = mu * e[3 + i];
        }
        double w[12];
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            w[n * 3 + 0] = g[n][0] * s[0] + g[n][1] * s[3] + g[n][2] * s[5];
            w[n * 3 + 1] = g[n][1] * s[1] + g[n][0] * s[3] + g[n][2] * s[4];
            w[n * 3 + 2] = g[n][2] * s[2] + g[n][1] * s[4] + g[n][0] * s[5];
        }
        double num = 0.0, den = 0.0, norm = 0.0;
#pragma unroll
        for (int i = 0; i < 12; ++i) {
            num += v[i] * w[i];
            den += v[i] * v[i];
            norm += w[i] * w[i];
        }
        const double next = den > 0.0 ? num / den : 0.0;
        norm = sqrt(norm);
        if (!(norm > 0.0)) {
            lam = 0.0;
            break;
        }
        if (SCALE_BY_RECIPROCAL) {
            const double inv = 1.0 / norm;
#pragma unroll
            for (int i = 0; i < 12; ++i) v[i] = w[i] * inv;
        } else {
#pragma unroll
            for (int i = 0; i < 12; ++i) v[i] = w[i] / norm;
        }
        if (it > 8 && fabs(next - lam) <= 1e-10 * fabs(next)) {
            lam = next;
            break;
        }
        lam = next;
    }
    return 4.0 / rho * lam;
}

}  // namespace fs
