// shell_setup.cu -- solid-shell rest forms, lumped mass, Gauss volumes and the
// element critical step, in FP64 on the device.
//
// Compiled with -fmad=false and written in the reference's operation order, so the
// double forms are the same bits solidshell::computeRestForms produces on the CPU
// (engine/sim/solid_shell.cpp:237-375), the lumped masses are elementMass's
// (:655-663), the Gauss volumes gaussVolumes's (:665-673) and the element step
// criticalTimestep's (:1088-1133).  One thread per element; the scratch (B in double,
// the condensed 24x24 stiffness) lives in local memory.  This is set-up work, run
// once per zone: it replaces the promotion cost the reference pays on the CPU
// (21.9 us per element per core, docs/07-fem-spike-findings.md:262).
#include "common.cuh"
#include "shell.hpp"

namespace fs {
namespace {

// elements per launch of the one-thread-per-element set-up (its stiffness scratch is
// 576 doubles x this many)
constexpr long long kSetupChunk = 1 << 16;
__device__ __constant__ double kXi[8] = {-1, +1, +1, -1, -1, +1, +1, -1};
__device__ __constant__ double kEta[8] = {-1, -1, +1, +1, -1, -1, +1, +1};
__device__ __constant__ double kZta[8] = {-1, -1, -1, -1, +1, +1, +1, +1};
__device__ __constant__ double kShearSample[4][2] = {{-1, 0}, {+1, 0}, {0, -1}, {0, +1}};
__device__ __constant__ double kCornerSample[4][2] = {{-1, -1}, {+1, -1}, {+1, +1}, {-1, +1}};

__device__ double det3(const double m[3][3]) {
    return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
           m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
}

// invert3, solid_shell.cpp:44-58
__device__ double inv3(const double m[3][3], double inv[3][3]) {
    const double det = det3(m);
    if (det == 0.0) return 0.0;
    const double d = 1.0 / det;
    inv[0][0] = (m[1][1] * m[2][2] - m[1][2] * m[2][1]) * d;
    inv[0][1] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) * d;
    inv[0][2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) * d;
    inv[1][0] = (m[1][2] * m[2][0] - m[1][0] * m[2][2]) * d;
    inv[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) * d;
    inv[1][2] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) * d;
    inv[2][0] = (m[1][0] * m[2][1] - m[1][1] * m[2][0]) * d;
    inv[2][1] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) * d;
    inv[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) * d;
    return det;
}

struct Point {
    double dn[8][3];
    double jac[3][3];
};

// evaluate, solid_shell.cpp:67-83
__device__ void evaluate(const double nodes[24], double xi, double eta, double zta, Point& p) {
    for (int a = 0; a < 8; ++a) {
        const double x = 1.0 + xi * kXi[a];
        const double y = 1.0 + eta * kEta[a];
        const double z = 1.0 + zta * kZta[a];
        p.dn[a][0] = 0.125 * kXi[a] * y * z;
        p.dn[a][1] = 0.125 * kEta[a] * x * z;
        p.dn[a][2] = 0.125 * kZta[a] * x * y;
    }
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) {
            double s = 0.0;
            for (int a = 0; a < 8; ++a) s += p.dn[a][k] * nodes[a * 3 + i];
            p.jac[i][k] = s;
        }
}

// one row of naturalB (solid_shell.cpp:92-106) for every DOF
__device__ void natural_b_row(const Point& p, int row, double out[24]) {
    for (int a = 0; a < 8; ++a)
        for (int i = 0; i < 3; ++i) {
            const double g0 = p.jac[i][0], g1 = p.jac[i][1], g2 = p.jac[i][2];
            const double n0 = p.dn[a][0], n1 = p.dn[a][1], n2 = p.dn[a][2];
            double v;
            switch (row) {
                case 0: v = n0 * g0; break;
                case 1: v = n1 * g1; break;
                case 2: v = n2 * g2; break;
                case 3: v = n1 * g0 + n0 * g1; break;
                case 4: v = n2 * g1 + n1 * g2; break;
                default: v = n0 * g2 + n2 * g0; break;
            }
            out[a * 3 + i] = v;
        }
}

// voigtTransform, solid_shell.cpp:114-144
__device__ void voigt_transform(const double a[3][3], double t[6][6]) {
    const int row[6] = {0, 1, 2, 0, 1, 2};
    const int col[6] = {0, 1, 2, 1, 2, 0};
    for (int j = 0; j < 6; ++j) {
        double e[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        const double v = j < 3 ? 1.0 : 0.5;
        e[row[j]][col[j]] = v;
        e[col[j]][row[j]] = v;
        double ea[3][3];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                double s = 0.0;
                for (int k = 0; k < 3; ++k) s += e[r][k] * a[k][c];
                ea[r][c] = s;
            }
        double m[3][3];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                double s = 0.0;
                for (int k = 0; k < 3; ++k) s += a[k][r] * ea[k][c];
                m[r][c] = s;
            }
        t[0][j] = m[0][0];
        t[1][j] = m[1][1];
        t[2][j] = m[2][2];
        t[3][j] = 2.0 * m[0][1];
        t[4][j] = 2.0 * m[1][2];
        t[5][j] = 2.0 * m[2][0];
    }
}

struct Forms {
    double b[8][6][24];
    double g[8][6][7];
    double w[8];
    double j0[9];
    int eas;
    int ok;
};

// computeForms, solid_shell.cpp:237-375.
__device__ void compute_forms(const double nodes[24], int formulation, Forms& f) {
    const bool ans = formulation >= 1, eas = formulation >= 2;
    f.eas = eas ? 7 : 0;
    f.ok = 1;
    Point centre;
    evaluate(nodes, 0.0, 0.0, 0.0, centre);
    double a0[3][3];
    const double det0 = inv3(centre.jac, a0);
    if (!(det0 > 0.0)) {
        f.ok = 0;
        return;
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) f.j0[i * 3 + j] = a0[i][j];
    double t0[6][6];
    voigt_transform(a0, t0);
    const double q = 1.0 / sqrt(3.0);
    double shear_s[2][4][24], thick_s[2][4][24];
    if (ans)
        for (int level = 0; level < 2; ++level) {
            const double zeta = level ? q : -q;
            for (int s = 0; s < 4; ++s) {
                Point p;
                evaluate(nodes, kShearSample[s][0], kShearSample[s][1], zeta, p);
                natural_b_row(p, s < 2 ? 4 : 5, shear_s[level][s]);
                evaluate(nodes, kCornerSample[s][0], kCornerSample[s][1], zeta, p);
                natural_b_row(p, 2, thick_s[level][s]);
            }
        }
    for (int gp = 0; gp < 8; ++gp) {
        const double xi = (gp & 1) ? q : -q;
        const double eta = (gp & 2) ? q : -q;
        const double zta = (gp & 4) ? q : -q;
        const int level = (gp & 4) ? 1 : 0;
        Point p;
        evaluate(nodes, xi, eta, zta, p);
        double a[3][3];
        const double det = inv3(p.jac, a);
        if (!(det > 0.0)) {
            f.ok = 0;
            return;
        }
        f.w[gp] = det;
        double bn[6][24];
        for (int r = 0; r < 6; ++r) natural_b_row(p, r, bn[r]);
        if (ans) {
            const double wa = 0.5 * (1.0 - xi), wc = 0.5 * (1.0 + xi);
            const double wb = 0.5 * (1.0 - eta), wd = 0.5 * (1.0 + eta);
            for (int c = 0; c < 24; ++c) {
                bn[4][c] = wa * shear_s[level][0][c] + wc * shear_s[level][1][c];
                bn[5][c] = wb * shear_s[level][2][c] + wd * shear_s[level][3][c];
            }
            for (int c = 0; c < 24; ++c) bn[2][c] = 0.0;
            for (int s = 0; s < 4; ++s) {
                const double w = 0.25 * (1.0 + xi * kCornerSample[s][0]) * (1.0 + eta * kCornerSample[s][1]);
                for (int c = 0; c < 24; ++c) bn[2][c] += w * thick_s[level][s][c];
            }
        }
        double t[6][6];
        voigt_transform(a, t);
        for (int i = 0; i < 6; ++i)
            for (int c = 0; c < 24; ++c) {
                double s = 0.0;
                for (int k = 0; k < 6; ++k) s += t[i][k] * bn[k][c];
                f.b[gp][i][c] = s;
            }
        if (!eas) {
            for (int i = 0; i < 6; ++i)
                for (int j = 0; j < 7; ++j) f.g[gp][i][j] = 0.0;
            continue;
        }
        // enhancedM (solid_shell.cpp:168-178): nonzeros m[0][0]=xi, m[1][1]=eta,
        // m[2][2]=zeta, m[2][3]=xi zeta, m[2][4]=eta zeta, m[3][5]=xi, m[3][6]=eta
        double m[6][7];
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 7; ++j) m[i][j] = 0.0;
        m[0][0] = xi;
        m[1][1] = eta;
        m[2][2] = zta;
        m[2][3] = xi * zta;
        m[2][4] = eta * zta;
        m[3][5] = xi;
        m[3][6] = eta;
        const double scale = det0 / det;
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 7; ++j) {
                double s = 0.0;
                for (int k = 0; k < 6; ++k) s += t0[i][k] * m[k][j];
                f.g[gp][i][j] = scale * s;
            }
    }
    if (eas)
        for (int j = 0; j < 7; ++j) {
            double norm = 0.0;
            for (int gp = 0; gp < 8; ++gp)
                for (int i = 0; i < 6; ++i) norm += f.w[gp] * f.g[gp][i][j] * f.g[gp][i][j];
            if (!(norm > 0.0)) continue;
            const double inverse = 1.0 / sqrt(norm);
            for (int gp = 0; gp < 8; ++gp)
                for (int i = 0; i < 6; ++i) f.g[gp][i][j] *= inverse;
        }
}

// solveSmall, solid_shell.cpp:432-457
__device__ bool solve_small(const double a[49], int n, double* rhs, int columns) {
    double l[49];
    for (int i = 0; i < 49; ++i) l[i] = 0.0;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j <= i; ++j) {
            double s = a[i * 7 + j];
            for (int k = 0; k < j; ++k) s -= l[i * 7 + k] * l[j * 7 + k];
            if (i == j) {
                if (!(s > 0.0)) return false;
                l[i * 7 + i] = sqrt(s);
            } else {
                l[i * 7 + j] = s / l[j * 7 + j];
            }
        }
    for (int c = 0; c < columns; ++c) {
        for (int i = 0; i < n; ++i) {
            double s = rhs[i * columns + c];
            for (int k = 0; k < i; ++k) s -= l[i * 7 + k] * rhs[k * columns + c];
            rhs[i * columns + c] = s / l[i * 7 + i];
        }
        for (int i = n - 1; i >= 0; --i) {
            double s = rhs[i * columns + c];
            for (int k = i + 1; k < n; ++k) s -= l[k * 7 + i] * rhs[k * columns + c];
            rhs[i * columns + c] = s / l[i * 7 + i];
        }
    }
    return true;
}

// elementStiffness from computed forms: computeBlocks (solid_shell.cpp:377-429) and
// the static condensation (:509-535).
// out holds the 576 entries at a stride (the scratch is entry-major across elements, so
// the threads of a warp touch adjacent words).
__device__ void stiffness(const Forms& f, double E, double nu, double* out /*576 x stride*/, size_t stride) {
    const double lambda = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double mu = E / (2.0 * (1.0 + nu));
    double c[6][6];
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) c[i][j] = 0.0;
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) c[i][j] = lambda;
        c[i][i] += 2.0 * mu;
        c[3 + i][3 + i] = mu;
    }
    double kua[24 * 7], kaa[49];
    for (int i = 0; i < 576; ++i) out[i * stride] = 0.0;
    for (int i = 0; i < 24 * 7; ++i) kua[i] = 0.0;
    for (int i = 0; i < 49; ++i) kaa[i] = 0.0;
    for (int gp = 0; gp < 8; ++gp) {
        const double w = f.w[gp];
        double cb[6][24];
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 24; ++j) {
                double s = 0.0;
                for (int k = 0; k < 6; ++k) s += c[i][k] * f.b[gp][k][j];
                cb[i][j] = s;
            }
        for (int i = 0; i < 24; ++i)
            for (int j = 0; j < 24; ++j) {
                double s = 0.0;
                for (int k = 0; k < 6; ++k) s += f.b[gp][k][i] * cb[k][j];
                out[(i * 24 + j) * stride] += w * s;
            }
        if (f.eas == 0) continue;
        double cg[6][7];
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 7; ++j) {
                double s = 0.0;
                for (int k = 0; k < 6; ++k) s += c[i][k] * f.g[gp][k][j];
                cg[i][j] = s;
            }
        for (int i = 0; i < 24; ++i)
            for (int j = 0; j < 7; ++j) {
                double s = 0.0;
                for (int k = 0; k < 6; ++k) s += f.b[gp][k][i] * cg[k][j];
                kua[i * 7 + j] += w * s;
            }
        for (int i = 0; i < 7; ++i)
            for (int j = 0; j < 7; ++j) {
                double s = 0.0;
                for (int k = 0; k < 6; ++k) s += f.g[gp][k][i] * cg[k][j];
                kaa[i * 7 + j] += w * s;
            }
    }
    if (f.eas == 0) return;
    double x[7 * 24];
    for (int i = 0; i < f.eas; ++i)
        for (int j = 0; j < 24; ++j) x[i * 24 + j] = kua[j * 7 + i];
    if (!solve_small(kaa, f.eas, x, 24)) return;
    for (int i = 0; i < 24; ++i)
        for (int j = 0; j < 24; ++j) {
            double s = 0.0;
            for (int k = 0; k < f.eas; ++k) s += kua[i * 7 + k] * x[k * 24 + j];
            out[(i * 24 + j) * stride] -= s;
        }
}

// criticalTimestep, solid_shell.cpp:1088-1133
__device__ double power_dt(const double* k, size_t stride, const double m[8], double safety) {
    for (int a = 0; a < 8; ++a)
        if (!(m[a] > 0.0)) return 0.0;
    double d[24];
    for (int a = 0; a < 8; ++a)
        for (int i = 0; i < 3; ++i) d[a * 3 + i] = 1.0 / sqrt(m[a]);
    double v[24];
    for (int i = 0; i < 24; ++i) v[i] = 1.0 + 0.37 * i - 0.11 * i * i;
    double lambda = 0.0;
    for (int it = 0; it < 400; ++it) {
        double w[24];
        for (int i = 0; i < 24; ++i) {
            double s = 0.0;
            for (int j = 0; j < 24; ++j) s += k[(i * 24 + j) * stride] * (d[j] * v[j]);
            w[i] = d[i] * s;
        }
        double num = 0.0, den = 0.0;
        for (int i = 0; i < 24; ++i) {
            num += v[i] * w[i];
            den += v[i] * v[i];
        }
        const double next = den > 0.0 ? num / den : 0.0;
        double norm = 0.0;
        for (int i = 0; i < 24; ++i) norm += w[i] * w[i];
        norm = sqrt(norm);
        if (!(norm > 0.0)) return 0.0;
        for (int i = 0; i < 24; ++i) v[i] = w[i] / norm;
        if (it > 8 && fabs(next - lambda) <= 1e-10 * fabs(next)) {
            lambda = next;
            break;
        }
        lambda = next;
    }
    if (!(lambda > 0.0)) return 0.0;
    return safety * 2.0 / sqrt(lambda);
}

__global__ void __launch_bounds__(64) shell_setup_kernel(ShellSetupArgs a, double* scratch_k) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= a.elements) return;
    double nodes[24];
    for (int n = 0; n < 8; ++n) {
        const uint32_t id = a.index[e * 8 + n];
        for (int i = 0; i < 3; ++i) nodes[n * 3 + i] = a.rest[(size_t)id * 3 + i];
    }
    Forms f;
    compute_forms(nodes, a.formulation, f);
    if (a.ok) a.ok[e] = f.ok;
    if (a.forms64) {
        double* o = a.forms64 + (size_t)e * 1507;
        for (int gp = 0; gp < 8; ++gp)
            for (int i = 0; i < 6; ++i) {
                for (int j = 0; j < 24; ++j) o[(gp * 6 + i) * 24 + j] = f.ok ? f.b[gp][i][j] : 0.0;
                for (int j = 0; j < 7; ++j) o[1152 + (gp * 6 + i) * 7 + j] = f.ok ? f.g[gp][i][j] : 0.0;
            }
        for (int gp = 0; gp < 8; ++gp) o[1488 + gp] = f.ok ? f.w[gp] : 0.0;
        for (int k = 0; k < 9; ++k) o[1496 + k] = f.ok ? f.j0[k] : 0.0;
        o[1505] = f.eas;
        o[1506] = f.ok;
    }
    if (a.gauss_volume || a.corner_mass || a.dt_out) {
        // gaussVolumes / elementMass (solid_shell.cpp:655-673) run computeForms with
        // the displacement formulation; its weights det J are the ones above (the
        // assumed-strain cures change B and G, never the Jacobian), so only the shape
        // functions at the Gauss points are new here.
        double m[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        const double q = 1.0 / sqrt(3.0);
        if (f.ok)
            for (int gp = 0; gp < 8; ++gp) {
                const double xi = (gp & 1) ? q : -q;
                const double eta = (gp & 2) ? q : -q;
                const double zta = (gp & 4) ? q : -q;
                for (int n = 0; n < 8; ++n) {
                    const double shape = 0.125 * (1.0 + xi * kXi[n]) * (1.0 + eta * kEta[n]) * (1.0 + zta * kZta[n]);
                    m[n] += a.density * f.w[gp] * shape;
                }
            }
        if (a.gauss_volume)
            for (int gp = 0; gp < 8; ++gp) a.gauss_volume[e * 8 + gp] = f.ok ? f.w[gp] : 0.0;
        if (a.corner_mass)
            for (int n = 0; n < 8; ++n) a.corner_mass[a.slot[e * 8 + n]] = m[n];
        if (a.dt_out) {
            double* k = scratch_k + e;  // entry-major: entry i of element e at i * chunk + e
            if (f.ok) {
                // criticalTimestep builds its own stiffness from the nodes (for the
                // solid-shell formulation, the same forms as above).
                stiffness(f, a.youngs, a.poisson, k, kSetupChunk);
                a.dt_out[e] = power_dt(k, kSetupChunk, m, a.safety);
            } else {
                a.dt_out[e] = 0.0;
            }
        }
    }
}

// The solver's set-up with 8 lanes per element (lane = Gauss point): the element row
// (J0^-1 and the enhanced modes' scales det J0 n_j), the lumped corner masses and the
// Gauss volumes.  Each lane runs compute_forms's operations for its own point in the
// same order, and the element-wide steps combine the lanes' values in the reference's
// point order through shuffles -- the EAS column norms (sum over points, then rows),
// the lumped mass (sum over points), and the element's validity (every point's
// det J > 0).  Bit-identical to shell_setup_kernel's values.
__global__ void __launch_bounds__(128) shell_setup_lanes(ShellSetupArgs a) {
    const int lane = threadIdx.x & 31, gp = lane & 7;
    const long long e_raw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 3;
    const bool valid = e_raw < a.elements;
    const long long e = valid ? e_raw : a.elements - 1;  // tail lanes shadow the last element, write nothing
    const unsigned group_mask = 0xffu << (lane & 24);
    double nodes[24];
    for (int n = 0; n < 8; ++n) {
        const uint32_t id = a.index[e * 8 + n];
        for (int i = 0; i < 3; ++i) nodes[n * 3 + i] = a.rest[(size_t)id * 3 + i];
    }
    const bool eas = a.formulation >= 2;
    Point centre;
    evaluate(nodes, 0.0, 0.0, 0.0, centre);
    double a0[3][3];
    const double det0 = inv3(centre.jac, a0);
    const double q = 1.0 / sqrt(3.0);
    const double xi = (gp & 1) ? q : -q;
    const double eta = (gp & 2) ? q : -q;
    const double zta = (gp & 4) ? q : -q;
    Point p;
    evaluate(nodes, xi, eta, zta, p);
    double am[3][3];
    const double det = inv3(p.jac, am);
    // computeForms gives up on the element at the first point with det J <= 0
    const bool ok = (__ballot_sync(0xffffffffu, det0 > 0.0 && det > 0.0) & group_mask) == group_mask;
    // G: enhancedM mapped by the centre transform and scaled by det J0 / det J, for the
    // modes' norms; the step re-forms G from J0^-1 and the scale det J0 / norm_j
    double g[6][7];
    {
        double t0[6][6];
        voigt_transform(a0, t0);
        double m[6][7];
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 7; ++j) m[i][j] = 0.0;
        m[0][0] = xi;
        m[1][1] = eta;
        m[2][2] = zta;
        m[2][3] = xi * zta;
        m[2][4] = eta * zta;
        m[3][5] = xi;
        m[3][6] = eta;
        const double scale = det0 / det;
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 7; ++j) {
                double sum = 0.0;
                for (int k = 0; k < 6; ++k) sum += t0[i][k] * m[k][j];
                g[i][j] = eas ? scale * sum : 0.0;
            }
    }
    double mine = 0.0;  // this lane's mode (gp < 7): det J0 / norm, or det J0 for an unused mode
    if (eas)
        for (int j = 0; j < 7; ++j) {
            // sum over points, then rows, in the reference's order, in every lane alike
            double norm = 0.0;
            for (int src = 0; src < 8; ++src)
                for (int i = 0; i < 6; ++i) {
                    const double term = __shfl_sync(0xffffffffu, det * g[i][j] * g[i][j], (lane & 24) + src);
                    norm += term;
                }
            const double inverse = norm > 0.0 ? 1.0 / sqrt(norm) : 1.0;  // an unused mode stays as it is
            if (j == gp) mine = det0 * inverse;
        }
    // lumped corner mass (elementMass, solid_shell.cpp:655-663): lane n sums node n over
    // the points in order
    double mass = 0.0;
    for (int src = 0; src < 8; ++src) {
        const double w = __shfl_sync(0xffffffffu, det, (lane & 24) + src);
        const double sx = (src & 1) ? q : -q, sy = (src & 2) ? q : -q, sz = (src & 4) ? q : -q;
        const double shape = 0.125 * (1.0 + sx * kXi[gp]) * (1.0 + sy * kEta[gp]) * (1.0 + sz * kZta[gp]);
        mass += a.density * w * shape;
    }
    if (!valid) return;
    if (a.elem) {
        float* row = reinterpret_cast<float*>(a.elem + e * kShellElemQ);
        row[gp] = ok ? (float)a0[gp / 3][gp % 3] : 0.0f;
        if (gp == 0) row[8] = ok ? (float)a0[2][2] : 0.0f;
        if (gp < 7) row[9 + gp] = ok ? (float)mine : 0.0f;
    }
    if (a.gauss_volume) a.gauss_volume[e * 8 + gp] = ok ? det : 0.0;
    if (a.corner_mass) a.corner_mass[a.slot[e * 8 + gp]] = ok ? mass : 0.0;
}

__global__ void shell_mass_kernel(long long nodes, const uint32_t* offset, const double* corner_mass, double* mass64,
                                  float* mass, float* inv_mass) {
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nodes) return;
    double s = 0.0;
    for (uint32_t k = offset[n]; k < offset[n + 1]; ++k) s += corner_mass[k];
    if (mass64) mass64[n] = s;
    mass[n] = (float)s;
    inv_mass[n] = s > 0.0 ? (float)(1.0 / s) : 0.0f;
}

}  // namespace

void launch_shell_setup(const ShellSetupArgs& a, cudaStream_t stream) {
    if (!a.dt_out && !a.forms64 && !a.ok) {
        // the solver's set-up: element rows, masses, Gauss volumes, 8 lanes per element
        shell_setup_lanes<<<blocks_for(a.elements * 8, 128), 128, 0, stream>>>(a);
        return;
    }
    double* scratch = nullptr;
    const long long chunk = kSetupChunk;
    if (a.dt_out) cudaMallocAsync(&scratch, (size_t)chunk * 576 * sizeof(double), stream);
    for (long long first = 0; first < a.elements; first += chunk) {
        ShellSetupArgs c = a;
        const long long n = a.elements - first < chunk ? a.elements - first : chunk;
        // offset every per-element pointer to this chunk; the element id inside the
        // kernel is chunk-relative, so the lane-record layout needs whole groups
        c.elements = n;
        c.index = a.index + first * 8;
        c.slot = a.slot + first * 8;
        if (a.gauss_volume) c.gauss_volume = a.gauss_volume + first * 8;
        if (a.dt_out) c.dt_out = a.dt_out + first;
        if (a.forms64) c.forms64 = a.forms64 + first * 1507;
        if (a.ok) c.ok = a.ok + first;
        shell_setup_kernel<<<blocks_for(n, 64), 64, 0, stream>>>(c, scratch);
    }
    if (scratch) cudaFreeAsync(scratch, stream);
}

void launch_shell_mass(long long nodes, const uint32_t* offset, const double* corner_mass, double* mass64,
                       float* mass, float* inv_mass, cudaStream_t stream) {
    shell_mass_kernel<<<blocks_for(nodes, 256), 256, 0, stream>>>(nodes, offset, corner_mass, mass64, mass,
                                                                   inv_mass);
}

}  // namespace fs
