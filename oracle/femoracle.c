/*
 * femoracle.c -- plain-C restatement of the reference's explicit FEM step.
 *
 * TEST INFRASTRUCTURE ONLY (see femoracle.h).  The product never links this.
 *
 * Each function cites the reference file:line whose algorithm it restates.  The
 * arithmetic is written in the same order as the reference on purpose: compiled with
 * the flags in oracle/Makefile (IEEE double/single, no contraction) the restatement
 * reproduces the compiled reference bit for bit, which is how it is pinned
 * (tests/test_oracle.py).
 */
#include "femoracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

static double dmax(double a, double b) { return a > b ? a : b; }
static double dmin(double a, double b) { return a < b ? a : b; }

/* =========================================================================
 * J2 point law: engine/sim/plasticity.cpp
 * ========================================================================= */

/* flowStress / flowSlope, plasticity.cpp:124-142 */
static double flow_stress(const double *mat, double eps_p) {
    const double p = dmax(0.0, eps_p);
    if (mat[5] == 0.0) return mat[2] + mat[3] * p;
    return mat[6] * pow(mat[7] + p, mat[8]);
}

static double flow_slope(const double *mat, double eps_p) {
    const double p = dmax(0.0, eps_p);
    if (mat[5] == 0.0) return mat[3];
    return mat[6] * mat[8] * pow(mat[7] + p, mat[8] - 1.0);
}

/* tensorNormSquared, plasticity.cpp:26-29 */
static double tensor_norm2(const double v[6]) {
    return v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + 2.0 * (v[3] * v[3] + v[4] * v[4] + v[5] * v[5]);
}

/* deviator / vonMises / meanStress / triaxiality, plasticity.cpp:270-293 */
static double von_mises(const double s[6]) {
    const double mean = (s[0] + s[1] + s[2]) / 3.0;
    double d[6];
    for (int i = 0; i < 3; ++i) {
        d[i] = s[i] - mean;
        d[3 + i] = s[3 + i];
    }
    return sqrt(1.5) * sqrt(tensor_norm2(d));
}

static double triaxiality(const double s[6]) {
    const double q = von_mises(s);
    return q > 0.0 ? ((s[0] + s[1] + s[2]) / 3.0) / q : 0.0;
}

/* triaxialityFactor, plasticity.cpp:171-174 */
static double triax_factor(const double *mat, double eta) {
    if (eta <= mat[13]) return INFINITY;
    return exp(-mat[11] * (eta - mat[12]));
}

/* symmetricEigen (Jacobi), plasticity.cpp:35-71, and maxPrincipalDirection :295-315 */
static void max_principal_direction(const double stress[6], double out[3]) {
    double a[3][3] = {{stress[0], stress[3], stress[5]},
                      {stress[3], stress[1], stress[4]},
                      {stress[5], stress[4], stress[2]}};
    double v[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) v[i][j] = (i == j) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 64; ++sweep) {
        const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        if (off <= 0.0) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                const double apq = a[p][q];
                if (apq == 0.0) continue;
                const double theta = (a[q][q] - a[p][p]) / (2.0 * apq);
                const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; ++k) {
                    const double akp = a[k][p], akq = a[k][q];
                    a[k][p] = c * akp - s * akq;
                    a[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; ++k) {
                    const double apk = a[p][k], aqk = a[q][k];
                    a[p][k] = c * apk - s * aqk;
                    a[q][k] = s * apk + c * aqk;
                }
                for (int k = 0; k < 3; ++k) {
                    const double vkp = v[k][p], vkq = v[k][q];
                    v[k][p] = c * vkp - s * vkq;
                    v[k][q] = s * vkp + c * vkq;
                }
            }
    }
    int best = 0;
    for (int i = 1; i < 3; ++i)
        if (a[i][i] > a[best][best]) best = i;
    for (int i = 0; i < 3; ++i) out[i] = v[i][best];
    double norm = sqrt(out[0] * out[0] + out[1] * out[1] + out[2] * out[2]);
    if (!(norm > 0.0)) {
        out[0] = 1.0;
        out[1] = out[2] = 0.0;
        return;
    }
    int largest = 0;
    for (int i = 1; i < 3; ++i)
        if (fabs(out[i]) > fabs(out[largest])) largest = i;
    if (out[largest] < 0.0) norm = -norm;
    for (int i = 0; i < 3; ++i) out[i] /= norm;
}

/* elasticModuli, plasticity.cpp:244-254 */
static void elastic_moduli(const double *mat, double c[36]) {
    const double e = mat[0], nu = mat[1];
    const double lambda = e * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double mu = e / (2.0 * (1.0 + nu));
    for (int i = 0; i < 36; ++i) c[i] = 0.0;
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) c[i * 6 + j] = lambda;
        c[i * 6 + i] += 2.0 * mu;
        c[(3 + i) * 6 + (3 + i)] = mu;
    }
}

/* update, plasticity.cpp:319-505: elastic predictor, radial return with the
 * bracketed Newton on the consistency condition, damage, algorithmic tangent. */
int or_plastic_update(const double *mat, double failure_strain, const double strain[6],
                      double state[OR_POINT_LEN], double stress[6], double *tangent,
                      double incr[OR_INCR_LEN]) {
    double inc[OR_INCR_LEN] = {0};
    if (state[14] != 0.0) {
        for (int i = 0; i < 6; ++i) stress[i] = 0.0;
        if (tangent)
            for (int i = 0; i < 36; ++i) tangent[i] = 0.0;
        if (incr) memcpy(incr, inc, sizeof(inc));
        return 0;
    }
    const double root23 = sqrt(2.0 / 3.0);
    const double mu = mat[0] / (2.0 * (1.0 + mat[1]));
    const double kappa = mat[0] / (3.0 * (1.0 - 2.0 * mat[1]));

    double elastic[6];
    for (int i = 0; i < 6; ++i) elastic[i] = strain[i] - state[i];
    const double volumetric = elastic[0] + elastic[1] + elastic[2];
    const double pressure = kappa * volumetric;
    double trial[6];
    for (int i = 0; i < 3; ++i) {
        trial[i] = 2.0 * mu * (elastic[i] - volumetric / 3.0);
        trial[3 + i] = mu * elastic[3 + i];
    }
    double relative[6];
    for (int i = 0; i < 6; ++i) relative[i] = trial[i] - state[6 + i];
    const double relative_norm = sqrt(tensor_norm2(relative));
    const double yield_radius = root23 * flow_stress(mat, state[12]);
    const double excess = relative_norm - yield_radius;

    if (!(excess > 0.0)) {
        for (int i = 0; i < 3; ++i) {
            stress[i] = pressure + trial[i];
            stress[3 + i] = trial[3 + i];
        }
        if (tangent) elastic_moduli(mat, tangent);
        inc[6] = von_mises(stress);
        inc[7] = triaxiality(stress);
        if (incr) memcpy(incr, inc, sizeof(inc));
        return 0;
    }

    const double kinematic = mat[4];
    const double linear_part = 2.0 * mu + (2.0 / 3.0) * kinematic;
    double lo = 0.0, hi = excess / linear_part;
    double gamma = hi;
    int iterations = 0;
    for (; iterations < 50; ++iterations) {
        const double accumulated = state[12] + root23 * gamma;
        const double residual = relative_norm - linear_part * gamma - root23 * flow_stress(mat, accumulated);
        if (residual > 0.0)
            lo = gamma;
        else
            hi = gamma;
        if (fabs(residual) <= 1e-14 * yield_radius) break;
        const double slope = -linear_part - (2.0 / 3.0) * flow_slope(mat, accumulated);
        double next = gamma - residual / slope;
        if (!(next > lo && next < hi)) next = 0.5 * (lo + hi);
        if (fabs(next - gamma) <= 1e-15 * gamma) {
            gamma = next;
            break;
        }
        gamma = next;
    }

    double direction[6];
    for (int i = 0; i < 6; ++i) direction[i] = relative[i] / relative_norm;
    double dp[6];
    for (int i = 0; i < 3; ++i) {
        dp[i] = gamma * direction[i];
        dp[3 + i] = 2.0 * gamma * direction[3 + i];
    }
    for (int i = 0; i < 3; ++i) {
        stress[i] = pressure + trial[i] - 2.0 * mu * gamma * direction[i];
        stress[3 + i] = trial[3 + i] - 2.0 * mu * gamma * direction[3 + i];
    }
    double back[6];
    for (int i = 0; i < 6; ++i) back[i] = state[6 + i] + (2.0 / 3.0) * kinematic * gamma * direction[i];
    double effective[6];
    for (int i = 0; i < 6; ++i) effective[i] = stress[i] - back[i];

    inc[0] = 1.0;
    inc[8] = iterations + 1;
    inc[2] = gamma;
    inc[3] = root23 * gamma;
    {
        double s = 0.0;
        for (int i = 0; i < 6; ++i) s += stress[i] * dp[i];
        inc[5] = s;
        s = 0.0;
        for (int i = 0; i < 6; ++i) s += effective[i] * dp[i];
        inc[4] = s;
    }
    for (int i = 0; i < 6; ++i) {
        state[i] += dp[i];
        state[6 + i] = back[i];
    }
    state[12] += inc[3];
    inc[6] = von_mises(stress);
    inc[7] = triaxiality(stress);

    const double critical = failure_strain * triax_factor(mat, inc[7]);
    if (critical > 0.0 && isfinite(critical)) state[13] += inc[3] / critical;
    if (state[13] >= 1.0) {
        double normal[3];
        state[13] = 1.0;
        state[14] = 1.0;
        inc[1] = 1.0;
        max_principal_direction(stress, normal);
        for (int i = 0; i < 6; ++i) stress[i] = 0.0;
        if (tangent)
            for (int i = 0; i < 36; ++i) tangent[i] = 0.0;
        if (incr) memcpy(incr, inc, sizeof(inc));
        return 1;
    }
    if (tangent) {
        const double theta = 1.0 - 2.0 * mu * gamma / relative_norm;
        const double plastic_modulus = flow_slope(mat, state[12]) + kinematic;
        const double theta_bar = 1.0 / (1.0 + plastic_modulus / (3.0 * mu)) - (1.0 - theta);
        for (int i = 0; i < 36; ++i) tangent[i] = 0.0;
        for (int i = 0; i < 3; ++i) {
            for (int j = 0; j < 3; ++j)
                tangent[i * 6 + j] = kappa + 2.0 * mu * theta * ((i == j ? 1.0 : 0.0) - 1.0 / 3.0);
            tangent[(3 + i) * 6 + (3 + i)] = mu * theta;
        }
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 6; ++j) tangent[i * 6 + j] -= 2.0 * mu * theta_bar * direction[i] * direction[j];
    }
    if (incr) memcpy(incr, inc, sizeof(inc));
    return 1;
}

/* =========================================================================
 * Linear tets: engine/sim/fem.cpp
 * ========================================================================= */

/* Column-major 3x3 in float (fem.cpp:10-56). */
typedef struct { float m[9]; } m3f;
#define F3(a, r, c) ((a).m[(c) * 3 + (r)])

static m3f m3f_mul(const m3f *a, const m3f *b) {
    m3f r;
    for (int c = 0; c < 3; ++c)
        for (int i = 0; i < 3; ++i) {
            float s = 0;
            for (int k = 0; k < 3; ++k) s += F3(*a, i, k) * F3(*b, k, c);
            F3(r, i, c) = s;
        }
    return r;
}

static m3f m3f_tr(const m3f *a) {
    m3f r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) F3(r, i, j) = F3(*a, j, i);
    return r;
}

static float m3f_det(const m3f *a) {
    return F3(*a, 0, 0) * (F3(*a, 1, 1) * F3(*a, 2, 2) - F3(*a, 1, 2) * F3(*a, 2, 1)) -
           F3(*a, 0, 1) * (F3(*a, 1, 0) * F3(*a, 2, 2) - F3(*a, 1, 2) * F3(*a, 2, 0)) +
           F3(*a, 0, 2) * (F3(*a, 1, 0) * F3(*a, 2, 1) - F3(*a, 1, 1) * F3(*a, 2, 0));
}

static m3f m3f_inv(const m3f *a) {
    const float det = m3f_det(a);
    const float id = fabsf(det) > 1e-30f ? 1.0f / det : 0.0f;
    m3f r;
    F3(r, 0, 0) = (F3(*a, 1, 1) * F3(*a, 2, 2) - F3(*a, 1, 2) * F3(*a, 2, 1)) * id;
    F3(r, 0, 1) = (F3(*a, 0, 2) * F3(*a, 2, 1) - F3(*a, 0, 1) * F3(*a, 2, 2)) * id;
    F3(r, 0, 2) = (F3(*a, 0, 1) * F3(*a, 1, 2) - F3(*a, 0, 2) * F3(*a, 1, 1)) * id;
    F3(r, 1, 0) = (F3(*a, 1, 2) * F3(*a, 2, 0) - F3(*a, 1, 0) * F3(*a, 2, 2)) * id;
    F3(r, 1, 1) = (F3(*a, 0, 0) * F3(*a, 2, 2) - F3(*a, 0, 2) * F3(*a, 2, 0)) * id;
    F3(r, 1, 2) = (F3(*a, 0, 2) * F3(*a, 1, 0) - F3(*a, 0, 0) * F3(*a, 1, 2)) * id;
    F3(r, 2, 0) = (F3(*a, 1, 0) * F3(*a, 2, 1) - F3(*a, 1, 1) * F3(*a, 2, 0)) * id;
    F3(r, 2, 1) = (F3(*a, 0, 1) * F3(*a, 2, 0) - F3(*a, 0, 0) * F3(*a, 2, 1)) * id;
    F3(r, 2, 2) = (F3(*a, 0, 0) * F3(*a, 1, 1) - F3(*a, 0, 1) * F3(*a, 1, 0)) * id;
    return r;
}

/* polarRotation, fem.cpp:62-69: four fixed Higham iterations. */
static m3f m3f_polar(const m3f *f) {
    m3f r = *f;
    for (int i = 0; i < 4; ++i) {
        const m3f inv = m3f_inv(&r);
        const m3f rit = m3f_tr(&inv);
        for (int k = 0; k < 9; ++k) r.m[k] = 0.5f * (r.m[k] + rit.m[k]);
    }
    return r;
}

void or_box_tet_sizes(int nx, int ny, int nz, size_t *nodes, size_t *tets) {
    *nodes = (size_t)(nx + 1) * (size_t)(ny + 1) * (size_t)(nz + 1);
    *tets = (size_t)nx * (size_t)ny * (size_t)nz * 6u;
}

/* makeBoxTetMesh, fem.cpp:217-263: grid nodes (k*sy+j)*sx+i, six Kuhn tets per
 * cell around the 0-7 diagonal, orientation fixed by swapping corners 1 and 2. */
void or_box_tet_mesh(float lx, float ly, float lz, int nx, int ny, int nz, float *position,
                     uint32_t *index) {
    const int sx = nx + 1, sy = ny + 1, sz = nz + 1;
#define NODE_AT(i, j, k) ((uint32_t)(((k) * sy + (j)) * sx + (i)))
    for (int k = 0; k < sz; ++k)
        for (int j = 0; j < sy; ++j)
            for (int i = 0; i < sx; ++i) {
                float *p = &position[(size_t)NODE_AT(i, j, k) * 3];
                p[0] = lx * (float)i / (float)nx;
                p[1] = ly * (float)j / (float)ny;
                p[2] = lz * (float)k / (float)nz;
            }
    static const int cell_tets[6][4] = {{0, 1, 3, 7}, {0, 1, 7, 5}, {0, 5, 7, 4},
                                        {0, 3, 2, 7}, {0, 2, 6, 7}, {0, 4, 6, 7}};
    size_t out = 0;
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                uint32_t corner[8];
                for (int c = 0; c < 8; ++c)
                    corner[c] = NODE_AT(i + (c & 1), j + ((c >> 1) & 1), k + ((c >> 2) & 1));
                for (int t = 0; t < 6; ++t) {
                    uint32_t v[4];
                    for (int c = 0; c < 4; ++c) v[c] = corner[cell_tets[t][c]];
                    m3f dm;
                    for (int c = 0; c < 3; ++c)
                        for (int a = 0; a < 3; ++a)
                            F3(dm, a, c) = position[(size_t)v[c + 1] * 3 + a] - position[(size_t)v[0] * 3 + a];
                    if (m3f_det(&dm) < 0) {
                        const uint32_t s = v[1];
                        v[1] = v[2];
                        v[2] = s;
                    }
                    for (int c = 0; c < 4; ++c) index[out * 4 + c] = v[c];
                    ++out;
                }
            }
#undef NODE_AT
}

static void build_csr(size_t nodes, size_t elements, int corners, const uint32_t *index,
                      uint32_t *offset, uint32_t *entry) {
    for (size_t n = 0; n <= nodes; ++n) offset[n] = 0;
    for (size_t e = 0; e < elements; ++e)
        for (int c = 0; c < corners; ++c) ++offset[index[e * corners + c] + 1];
    for (size_t n = 0; n < nodes; ++n) offset[n + 1] += offset[n];
    uint32_t *cursor = (uint32_t *)malloc(sizeof(uint32_t) * (nodes ? nodes : 1));
    memcpy(cursor, offset, sizeof(uint32_t) * nodes);
    for (size_t e = 0; e < elements; ++e)
        for (int c = 0; c < corners; ++c)
            entry[cursor[index[e * corners + c]]++] = (uint32_t)e * (uint32_t)corners + (uint32_t)c;
    free(cursor);
}

/* computeRestState, fem.cpp:119-158 */
void or_tet32_rest_state(or_tet32 *m, float E, float nu, float rho) {
    (void)E;
    (void)nu;
    for (size_t n = 0; n < m->nodes * 3; ++n) m->velocity[n] = 0.0f;
    for (size_t n = 0; n < m->nodes; ++n) m->mass[n] = 0.0f;
    for (size_t t = 0; t < m->tets * 12; ++t) m->tet_force[t] = 0.0f;
    for (size_t t = 0; t < m->tets; ++t) {
        const uint32_t *idx = &m->index[t * 4];
        m3f dm;
        for (int c = 0; c < 3; ++c)
            for (int a = 0; a < 3; ++a)
                F3(dm, a, c) = m->position[(size_t)idx[c + 1] * 3 + a] - m->position[(size_t)idx[0] * 3 + a];
        const float volume = m3f_det(&dm) / 6.0f;
        m->rest_volume[t] = fabsf(volume);
        const m3f inv = m3f_inv(&dm);
        for (int k = 0; k < 9; ++k) m->rest_inv[t * 9 + k] = inv.m[k];
        const float quarter = rho * m->rest_volume[t] * 0.25f;
        for (int c = 0; c < 4; ++c) m->mass[idx[c]] += quarter;
    }
    build_csr(m->nodes, m->tets, 4, m->index, m->adj_offset, m->adj_entry);
}

/* tetForces, fem.cpp:73-117 */
void or_tet32_forces(const or_tet32 *m, size_t t, float lambda, float mu, float out[12]) {
    const uint32_t *idx = &m->index[t * 4];
    const float *p = m->position;
    m3f ds, dm_inv;
    for (int c = 0; c < 3; ++c)
        for (int a = 0; a < 3; ++a) F3(ds, a, c) = p[(size_t)idx[c + 1] * 3 + a] - p[(size_t)idx[0] * 3 + a];
    for (int k = 0; k < 9; ++k) dm_inv.m[k] = m->rest_inv[t * 9 + k];
    const m3f f = m3f_mul(&ds, &dm_inv);
    const m3f r = m3f_polar(&f);
    const m3f rt = m3f_tr(&r);
    const m3f s = m3f_mul(&rt, &f);
    m3f strain;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) F3(strain, i, j) = 0.5f * (F3(s, i, j) + F3(s, j, i));
    for (int i = 0; i < 3; ++i) F3(strain, i, i) -= 1.0f;
    const float trace = F3(strain, 0, 0) + F3(strain, 1, 1) + F3(strain, 2, 2);
    m3f stress;
    for (int k = 0; k < 9; ++k) stress.m[k] = 2.0f * mu * strain.m[k];
    for (int i = 0; i < 3; ++i) F3(stress, i, i) += lambda * trace;
    const m3f piola = m3f_mul(&r, &stress);
    const m3f dmt = m3f_tr(&dm_inv);
    const m3f h = m3f_mul(&piola, &dmt);
    const float scale = -m->rest_volume[t];
    float f0[3] = {0, 0, 0};
    for (int c = 0; c < 3; ++c)
        for (int a = 0; a < 3; ++a) {
            const float v = scale * F3(h, a, c);
            out[(c + 1) * 3 + a] = v;
            f0[a] -= v;
        }
    for (int a = 0; a < 3; ++a) out[a] = f0[a];
}

/* stepCpu, fem.cpp:187-215 */
void or_tet32_step(or_tet32 *m, float E, float nu, float rho, float dt, float gravity,
                   float damping, int steps) {
    (void)rho;
    const float lambda = E * nu / ((1.0f + nu) * (1.0f - 2.0f * nu));
    const float mu = E / (2.0f * (1.0f + nu));
    for (int s = 0; s < steps; ++s) {
        for (size_t t = 0; t < m->tets; ++t) or_tet32_forces(m, t, lambda, mu, &m->tet_force[t * 12]);
        for (size_t n = 0; n < m->nodes; ++n) {
            if (m->fixed[n]) {
                for (int k = 0; k < 3; ++k) m->velocity[n * 3 + k] = 0.0f;
                continue;
            }
            float force[3] = {0.0f, 0.0f, -gravity * m->mass[n]};
            for (uint32_t e = m->adj_offset[n]; e < m->adj_offset[n + 1]; ++e) {
                const uint32_t entry = m->adj_entry[e];
                const float *f = &m->tet_force[(size_t)(entry >> 2) * 12 + (entry & 3u) * 3];
                for (int k = 0; k < 3; ++k) force[k] += f[k];
            }
            const float inv_mass = 1.0f / m->mass[n];
            for (int k = 0; k < 3; ++k) {
                float v = m->velocity[n * 3 + k] + force[k] * inv_mass * dt;
                v *= damping;
                m->velocity[n * 3 + k] = v;
                m->position[n * 3 + k] += v * dt;
            }
        }
    }
}

/* shortestEdge / criticalTimestep, fem.cpp:160-185 */
float or_tet32_critical_dt(const or_tet32 *m, float E, float nu, float rho, float safety) {
    (void)nu;
    float shortest = INFINITY;
    for (size_t t = 0; t < m->tets; ++t) {
        const uint32_t *idx = &m->index[t * 4];
        for (int a = 0; a < 4; ++a)
            for (int b = a + 1; b < 4; ++b) {
                float d2 = 0;
                for (int k = 0; k < 3; ++k) {
                    const float d = m->position[(size_t)idx[a] * 3 + k] - m->position[(size_t)idx[b] * 3 + k];
                    d2 += d * d;
                }
                const float len = sqrtf(d2);
                shortest = shortest < len ? shortest : len;
            }
    }
    return safety * shortest / sqrtf(E / rho);
}

/* ---- the J2 tet in double (O-tet64) ------------------------------------- */

typedef struct { double m[9]; } m3d;
#define D3(a, r, c) ((a).m[(c) * 3 + (r)])

static m3d m3d_mul(const m3d *a, const m3d *b) {
    m3d r;
    for (int c = 0; c < 3; ++c)
        for (int i = 0; i < 3; ++i) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += D3(*a, i, k) * D3(*b, k, c);
            D3(r, i, c) = s;
        }
    return r;
}

static m3d m3d_tr(const m3d *a) {
    m3d r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) D3(r, i, j) = D3(*a, j, i);
    return r;
}

static double m3d_det(const m3d *a) {
    return D3(*a, 0, 0) * (D3(*a, 1, 1) * D3(*a, 2, 2) - D3(*a, 1, 2) * D3(*a, 2, 1)) -
           D3(*a, 0, 1) * (D3(*a, 1, 0) * D3(*a, 2, 2) - D3(*a, 1, 2) * D3(*a, 2, 0)) +
           D3(*a, 0, 2) * (D3(*a, 1, 0) * D3(*a, 2, 1) - D3(*a, 1, 1) * D3(*a, 2, 0));
}

static m3d m3d_inv(const m3d *a) {
    const double det = m3d_det(a);
    const double id = fabs(det) > 1e-300 ? 1.0 / det : 0.0;
    m3d r;
    D3(r, 0, 0) = (D3(*a, 1, 1) * D3(*a, 2, 2) - D3(*a, 1, 2) * D3(*a, 2, 1)) * id;
    D3(r, 0, 1) = (D3(*a, 0, 2) * D3(*a, 2, 1) - D3(*a, 0, 1) * D3(*a, 2, 2)) * id;
    D3(r, 0, 2) = (D3(*a, 0, 1) * D3(*a, 1, 2) - D3(*a, 0, 2) * D3(*a, 1, 1)) * id;
    D3(r, 1, 0) = (D3(*a, 1, 2) * D3(*a, 2, 0) - D3(*a, 1, 0) * D3(*a, 2, 2)) * id;
    D3(r, 1, 1) = (D3(*a, 0, 0) * D3(*a, 2, 2) - D3(*a, 0, 2) * D3(*a, 2, 0)) * id;
    D3(r, 1, 2) = (D3(*a, 0, 2) * D3(*a, 1, 0) - D3(*a, 0, 0) * D3(*a, 1, 2)) * id;
    D3(r, 2, 0) = (D3(*a, 1, 0) * D3(*a, 2, 1) - D3(*a, 1, 1) * D3(*a, 2, 0)) * id;
    D3(r, 2, 1) = (D3(*a, 0, 1) * D3(*a, 2, 0) - D3(*a, 0, 0) * D3(*a, 2, 1)) * id;
    D3(r, 2, 2) = (D3(*a, 0, 0) * D3(*a, 1, 1) - D3(*a, 0, 1) * D3(*a, 1, 0)) * id;
    return r;
}

/* Higham iteration: fixed count as fem.cpp:62, or to convergence as
 * solid_shell.cpp:473-487 (step < 1e-16, at most 64). */
static m3d m3d_polar(const m3d *f, int fixed) {
    m3d r = *f;
    const int limit = fixed > 0 ? fixed : 64;
    for (int it = 0; it < limit; ++it) {
        if (fixed <= 0 && m3d_det(&r) == 0.0) return r;
        const m3d inv = m3d_inv(&r);
        const m3d rit = m3d_tr(&inv);
        double worst = 0;
        for (int k = 0; k < 9; ++k) {
            const double next = 0.5 * (r.m[k] + rit.m[k]);
            worst = dmax(worst, fabs(next - r.m[k]));
            r.m[k] = next;
        }
        if (fixed <= 0 && worst < 1e-16) return r;
    }
    return r;
}

/* computeRestState (fem.cpp:119-158) in double. */
void or_tet64_rest_state(or_tet64 *m, double rho) {
    for (size_t n = 0; n < m->nodes; ++n) m->mass[n] = 0.0;
    for (size_t t = 0; t < m->tets; ++t) {
        const uint32_t *idx = &m->index[t * 4];
        m3d dm;
        for (int c = 0; c < 3; ++c)
            for (int a = 0; a < 3; ++a)
                D3(dm, a, c) = m->position[(size_t)idx[c + 1] * 3 + a] - m->position[(size_t)idx[0] * 3 + a];
        const double volume = m3d_det(&dm) / 6.0;
        m->rest_volume[t] = fabs(volume);
        const m3d inv = m3d_inv(&dm);
        for (int k = 0; k < 9; ++k) m->rest_inv[t * 9 + k] = inv.m[k];
        const double quarter = rho * m->rest_volume[t] * 0.25;
        for (int c = 0; c < 4; ++c) m->mass[idx[c]] += quarter;
    }
    build_csr(m->nodes, m->tets, 4, m->index, m->adj_offset, m->adj_entry);
}

/* The element part of one O-tet64 step for tet t: fem.cpp:73-117 in double with the
 * J2 point law at the single point.  Writes the tet's corner forces and stress, its
 * plastic state, and its dissipation and strain energy into diss[t] and energy[t]. */
static void tet64_element(or_tet64 *m, const or_tet64_params *p, const double *mat, double mu, double bulk,
                          size_t t, double *diss, double *energy) {
    const uint32_t *idx = &m->index[t * 4];
    const double *x = m->position;
    m3d ds, dm_inv;
    for (int c = 0; c < 3; ++c)
        for (int a = 0; a < 3; ++a) D3(ds, a, c) = x[(size_t)idx[c + 1] * 3 + a] - x[(size_t)idx[0] * 3 + a];
    for (int k = 0; k < 9; ++k) dm_inv.m[k] = m->rest_inv[t * 9 + k];
    const m3d f = m3d_mul(&ds, &dm_inv);
    const m3d r = m3d_polar(&f, p->polar_fixed);
    const m3d rt = m3d_tr(&r);
    const m3d sm = m3d_mul(&rt, &f);
    double strain[6];
    strain[0] = 0.5 * (D3(sm, 0, 0) + D3(sm, 0, 0)) - 1.0;
    strain[1] = 0.5 * (D3(sm, 1, 1) + D3(sm, 1, 1)) - 1.0;
    strain[2] = 0.5 * (D3(sm, 2, 2) + D3(sm, 2, 2)) - 1.0;
    strain[3] = 2.0 * (0.5 * (D3(sm, 0, 1) + D3(sm, 1, 0)));
    strain[4] = 2.0 * (0.5 * (D3(sm, 1, 2) + D3(sm, 2, 1)));
    strain[5] = 2.0 * (0.5 * (D3(sm, 2, 0) + D3(sm, 0, 2)));
    double point[OR_POINT_LEN] = {0};
    double *ps = &m->plastic[t * 7];
    for (int i = 0; i < 6; ++i) point[i] = ps[i];
    point[12] = ps[6];
    double sv[6], inc[OR_INCR_LEN];
    or_plastic_update(mat, INFINITY, strain, point, sv, NULL, inc);
    for (int i = 0; i < 6; ++i) ps[i] = point[i];
    ps[6] = point[12];
    for (int i = 0; i < 6; ++i) m->stress[t * 6 + i] = sv[i];
    const double vol = m->rest_volume[t];
    diss[t] = vol * inc[4];
    const double pressure = (sv[0] + sv[1] + sv[2]) / 3.0;
    double density = 0;
    for (int i = 0; i < 3; ++i) density += 0.5 * sv[i] * ((sv[i] - pressure) / (2.0 * mu) + pressure / (3.0 * bulk));
    for (int i = 3; i < 6; ++i) density += 0.5 * sv[i] * (sv[i] / mu);
    energy[t] = vol * density;

    m3d stress;
    D3(stress, 0, 0) = sv[0];
    D3(stress, 1, 1) = sv[1];
    D3(stress, 2, 2) = sv[2];
    D3(stress, 0, 1) = D3(stress, 1, 0) = sv[3];
    D3(stress, 1, 2) = D3(stress, 2, 1) = sv[4];
    D3(stress, 2, 0) = D3(stress, 0, 2) = sv[5];
    const m3d piola = m3d_mul(&r, &stress);
    const m3d dmt = m3d_tr(&dm_inv);
    const m3d h = m3d_mul(&piola, &dmt);
    const double scale = -vol;
    double *out = &m->tet_force[t * 12];
    double f0[3] = {0, 0, 0};
    for (int c = 0; c < 3; ++c)
        for (int a = 0; a < 3; ++a) {
            const double v = scale * D3(h, a, c);
            out[(c + 1) * 3 + a] = v;
            f0[a] -= v;
        }
    for (int a = 0; a < 3; ++a) out[a] = f0[a];
}

#define OR_MAX_THREADS 256

/* The node part of one O-tet64 step for node n (fem.cpp:196-214, the ramped external
 * load added after the gather): its velocity and position, and its contributions to
 * the external work (per DOF), the kinetic energy (per DOF) and gravity's work. */
static void tet64_node(or_tet64 *m, const or_tet64_params *p, double lf, size_t n, double *nw, double *nk,
                       double *ng) {
    if (m->fixed[n]) {
        for (int k = 0; k < 3; ++k) m->velocity[n * 3 + k] = 0.0;
        return;
    }
    double force[3] = {0.0, 0.0, -p->gravity * m->mass[n]};
    for (uint32_t e = m->adj_offset[n]; e < m->adj_offset[n + 1]; ++e) {
        const uint32_t entry = m->adj_entry[e];
        const double *fs = &m->tet_force[(size_t)(entry >> 2) * 12 + (entry & 3u) * 3];
        for (int k = 0; k < 3; ++k) force[k] += fs[k];
    }
    double ext[3] = {0.0, 0.0, 0.0};
    if (m->fext)
        for (int k = 0; k < 3; ++k) ext[k] = lf * m->fext[n * 3 + k];
    for (int k = 0; k < 3; ++k) force[k] += ext[k];
    const double inv_mass = 1.0 / m->mass[n];
    for (int k = 0; k < 3; ++k) {
        double v = m->velocity[n * 3 + k] + force[k] * inv_mass * p->dt;
        v *= p->damping;
        m->velocity[n * 3 + k] = v;
        m->position[n * 3 + k] += v * p->dt;
        nw[n * 3 + k] = ext[k] * v * p->dt;
        nk[n * 3 + k] = 0.5 * m->mass[n] * v * v;
    }
    ng[n] = -p->gravity * m->mass[n] * m->velocity[n * 3 + 2] * p->dt;
}

typedef struct {
    or_tet64 *m;
    const or_tet64_params *p;
    const double *mat;
    double mu, bulk, lf;
    size_t begin, end;
    double *diss, *energy, *nw, *nk, *ng;
    int nodes; /* 0: tets [begin, end); 1: nodes [begin, end) */
} tet64_range;

static void *tet64_range_run(void *arg) {
    const tet64_range *r = (const tet64_range *)arg;
    for (size_t i = r->begin; i < r->end; ++i) {
        if (r->nodes)
            tet64_node(r->m, r->p, r->lf, i, r->nw, r->nk, r->ng);
        else
            tet64_element(r->m, r->p, r->mat, r->mu, r->bulk, i, r->diss, r->energy);
    }
    return NULL;
}

/* The element loop (nodes = 0) or the node loop (nodes = 1) of one step, over
 * `threads` host threads in contiguous ranges, or serially. */
static void tet64_loop(or_tet64 *m, const or_tet64_params *p, const double *mat, double mu, double bulk, double lf,
                       int threads, double *diss, double *energy, double *nw, double *nk, double *ng, int nodes) {
    const size_t count = nodes ? m->nodes : m->tets;
    const int n = threads < 1 ? 1 : (threads < OR_MAX_THREADS ? threads : OR_MAX_THREADS);
    tet64_range job[OR_MAX_THREADS];
    pthread_t tid[OR_MAX_THREADS];
    for (int k = 0; k < n; ++k)
        job[k] = (tet64_range){m, p, mat, mu, bulk, lf, count * k / n, count * (k + 1) / n, diss, energy, nw, nk, ng,
                               nodes};
    if (n == 1) {
        tet64_range_run(&job[0]);
        return;
    }
    for (int k = 0; k < n; ++k)
        if (pthread_create(&tid[k], NULL, tet64_range_run, &job[k])) abort();
    for (int k = 0; k < n; ++k) pthread_join(tid[k], NULL);
}

/* Steps of O-tet64: the element loop (tet64_element), then the node loop
 * (tet64_node), each over `threads` host threads when threads > 1.  The per-tet and
 * per-node energy terms are summed afterwards in tet and node order, as the serial
 * loops add them, so every thread count gives the same bits. */
static void tet64_steps(or_tet64 *m, const or_tet64_params *p, int steps, int threads) {
    double mat[OR_MAT_LEN] = {0};
    mat[0] = p->E;
    mat[1] = p->nu;
    mat[2] = p->yield;
    mat[3] = p->hardening;
    const double mu = p->E / (2.0 * (1.0 + p->nu));
    const double bulk = p->E / (3.0 * (1.0 - 2.0 * p->nu));
    double *diss = malloc((m->tets + 1) * sizeof(double));
    double *energy = malloc((m->tets + 1) * sizeof(double));
    double *nw = malloc((m->nodes * 3 + 1) * sizeof(double));
    double *nk = malloc((m->nodes * 3 + 1) * sizeof(double));
    double *ng = malloc((m->nodes + 1) * sizeof(double));
    if (!diss || !energy || !nw || !nk || !ng) abort();
    for (int s = 0; s < steps; ++s) {
        const double lf = p->ramp_steps > 0 ? dmin((double)(m->step + 1) / (double)p->ramp_steps, 1.0) : 1.0;
        tet64_loop(m, p, mat, mu, bulk, lf, threads, diss, energy, nw, nk, ng, 0);
        tet64_loop(m, p, mat, mu, bulk, lf, threads, diss, energy, nw, nk, ng, 1);
        /* the energy terms in node order, DOF by DOF, as the serial loop adds them */
        double work = 0.0, gwork = 0.0, kinetic = 0.0;
        for (size_t n = 0; n < m->nodes; ++n) {
            if (m->fixed[n]) continue;
            for (int k = 0; k < 3; ++k) {
                work += nw[n * 3 + k];
                kinetic += nk[n * 3 + k];
            }
            gwork += ng[n];
        }
        m->energy[0] += work;
        double dissipation = 0.0, strain_energy = 0.0;
        for (size_t t = 0; t < m->tets; ++t) {
            dissipation += diss[t];
            strain_energy += energy[t];
        }
        m->energy[1] += dissipation;
        m->energy[2] = strain_energy;
        m->energy[3] = kinetic;
        m->energy[4] += gwork;
        ++m->step;
    }
    free(diss);
    free(energy);
    free(nw);
    free(nk);
    free(ng);
}

/* Steps of O-tet64, serial. */
void or_tet64_step(or_tet64 *m, const or_tet64_params *p, int steps) { tet64_steps(m, p, steps, 1); }

/* The same steps with the element loop over `threads` host threads: bit-identical to
 * or_tet64_step, for the larger meshes the GPU tests check. */
void or_tet64_step_threads(or_tet64 *m, const or_tet64_params *p, int steps, int threads) {
    tet64_steps(m, p, steps, threads);
}

/* Element eigenvalue bound for a lumped-mass linear tet.  The element's mass matrix
 * is (rho V / 4) I and its stiffness V B^T C B, so omega_e^2 = (4/rho) lambda_max(B^T
 * C B); by the element eigenvalue theorem max_e omega_e^2 bounds the assembled
 * problem's.  Power iteration as solid_shell.cpp:1088-1133 (Rayleigh quotient, at
 * most 400 iterations, relative tolerance 1e-10, the same start vector). */
static double tet_omega2(const double *dm_inv, double E, double nu, double rho) {
    const double lambda = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double mu = E / (2.0 * (1.0 + nu));
    /* shape gradients: node c+1 -> row c of Dm^-1 (dm_inv column-major), node 0 = -sum */
    double g[4][3];
    for (int c = 0; c < 3; ++c)
        for (int a = 0; a < 3; ++a) g[c + 1][a] = dm_inv[a * 3 + c];
    for (int a = 0; a < 3; ++a) g[0][a] = -(g[1][a] + g[2][a] + g[3][a]);
    double v[12];
    for (int i = 0; i < 12; ++i) v[i] = 1.0 + 0.37 * i - 0.11 * i * i;
    double lam = 0.0;
    for (int it = 0; it < 400; ++it) {
        /* strain = B v (engineering shear) */
        double e[6] = {0, 0, 0, 0, 0, 0};
        for (int n = 0; n < 4; ++n) {
            const double *u = &v[n * 3];
            e[0] += g[n][0] * u[0];
            e[1] += g[n][1] * u[1];
            e[2] += g[n][2] * u[2];
            e[3] += g[n][1] * u[0] + g[n][0] * u[1];
            e[4] += g[n][2] * u[1] + g[n][1] * u[2];
            e[5] += g[n][0] * u[2] + g[n][2] * u[0];
        }
        const double tr = e[0] + e[1] + e[2];
        double s[6];
        for (int i = 0; i < 3; ++i) {
            s[i] = lambda * tr + 2.0 * mu * e[i];
            s[3 + i] = mu * e[3 + i];
        }
        double w[12];
        for (int n = 0; n < 4; ++n) {
            w[n * 3 + 0] = g[n][0] * s[0] + g[n][1] * s[3] + g[n][2] * s[5];
            w[n * 3 + 1] = g[n][1] * s[1] + g[n][0] * s[3] + g[n][2] * s[4];
            w[n * 3 + 2] = g[n][2] * s[2] + g[n][1] * s[4] + g[n][0] * s[5];
        }
        double num = 0.0, den = 0.0, norm = 0.0;
        for (int i = 0; i < 12; ++i) {
            num += v[i] * w[i];
            den += v[i] * v[i];
            norm += w[i] * w[i];
        }
        const double next = den > 0.0 ? num / den : 0.0;
        norm = sqrt(norm);
        if (!(norm > 0.0)) return 0.0;
        for (int i = 0; i < 12; ++i) v[i] = w[i] / norm;
        if (it > 8 && fabs(next - lam) <= 1e-10 * fabs(next)) {
            lam = next;
            break;
        }
        lam = next;
    }
    return 4.0 / rho * lam;
}

double or_tet64_critical_dt(const or_tet64 *m, double E, double nu, double rho, double safety) {
    double worst = 0.0;
    for (size_t t = 0; t < m->tets; ++t) worst = dmax(worst, tet_omega2(&m->rest_inv[t * 9], E, nu, rho));
    return worst > 0.0 ? safety * 2.0 / sqrt(worst) : 0.0;
}

/* =========================================================================
 * Solid-shell: engine/sim/solid_shell.cpp
 * ========================================================================= */

static const double kXi[8] = {-1, +1, +1, -1, -1, +1, +1, -1};
static const double kEta[8] = {-1, -1, +1, +1, -1, -1, +1, +1};
static const double kZta[8] = {-1, -1, -1, -1, +1, +1, +1, +1};

static double det3(const double m[3][3]) {
    return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
           m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
}

/* invert3, solid_shell.cpp:44-58 */
static double inv3(const double m[3][3], double inv[3][3]) {
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

typedef struct {
    double dn[8][3];
    double jac[3][3];
} point_t;

/* evaluate, solid_shell.cpp:67-83 */
static void evaluate(const double nodes[24], double xi, double eta, double zta, point_t *p) {
    for (int a = 0; a < 8; ++a) {
        const double x = 1.0 + xi * kXi[a];
        const double y = 1.0 + eta * kEta[a];
        const double z = 1.0 + zta * kZta[a];
        p->dn[a][0] = 0.125 * kXi[a] * y * z;
        p->dn[a][1] = 0.125 * kEta[a] * x * z;
        p->dn[a][2] = 0.125 * kZta[a] * x * y;
    }
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) {
            double s = 0.0;
            for (int a = 0; a < 8; ++a) s += p->dn[a][k] * nodes[a * 3 + i];
            p->jac[i][k] = s;
        }
}

/* naturalB, solid_shell.cpp:92-106 */
static void natural_b(const point_t *p, double b[6][24]) {
    for (int a = 0; a < 8; ++a)
        for (int i = 0; i < 3; ++i) {
            const int c = a * 3 + i;
            const double g0 = p->jac[i][0], g1 = p->jac[i][1], g2 = p->jac[i][2];
            const double n0 = p->dn[a][0], n1 = p->dn[a][1], n2 = p->dn[a][2];
            b[0][c] = n0 * g0;
            b[1][c] = n1 * g1;
            b[2][c] = n2 * g2;
            b[3][c] = n1 * g0 + n0 * g1;
            b[4][c] = n2 * g1 + n1 * g2;
            b[5][c] = n0 * g2 + n2 * g0;
        }
}

/* voigtTransform, solid_shell.cpp:114-144: natural -> Cartesian strain, eps = A^T E A */
static void voigt_transform(const double a[3][3], double t[6][6]) {
    static const int row[6] = {0, 1, 2, 0, 1, 2};
    static const int col[6] = {0, 1, 2, 1, 2, 0};
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

/* enhancedM, solid_shell.cpp:168-178: the seven EAS modes in natural components */
static void enhanced_m(double xi, double eta, double zta, double m[6][7]) {
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 7; ++j) m[i][j] = 0.0;
    m[0][0] = xi;
    m[1][1] = eta;
    m[2][2] = zta;
    m[2][3] = xi * zta;
    m[2][4] = eta * zta;
    m[3][5] = xi;
    m[3][6] = eta;
}

static const double kShearSample[4][2] = {{-1, 0}, {+1, 0}, {0, -1}, {0, +1}};
static const double kCornerSample[4][2] = {{-1, -1}, {+1, -1}, {+1, +1}, {-1, +1}};

/* computeForms, solid_shell.cpp:237-375: B after ANS (Dvorkin-Bathe shear,
 * Betsch-Stein thickness), G with the Simo-Rifai det J0/det J scaling, Gauss weights,
 * J0^-1; then the enhanced modes normalised in the weighted L2 norm.  `shape`
 * (may be NULL) receives N_a at the Gauss points for elementMass. */
static void compute_forms(const double nodes[24], int formulation, double *out, double shape[8][8]) {
    const int ans_shear = formulation >= 1, ans_thick = formulation >= 1, eas = formulation >= 2;
    double *B = out, *G = out + 1152, *W = out + 1488, *J0 = out + 1496;
    out[1505] = eas ? 7 : 0;
    out[1506] = 1.0;
    point_t centre;
    evaluate(nodes, 0.0, 0.0, 0.0, &centre);
    double a0[3][3];
    const double det0 = inv3(centre.jac, a0);
    if (!(det0 > 0.0)) {
        out[1506] = 0.0;
        return;
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) J0[i * 3 + j] = a0[i][j];
    double t0[6][6];
    voigt_transform(a0, t0);

    const double q = 1.0 / sqrt(3.0);
    static double shear_s[2][4][24], thick_s[2][4][24];
    memset(shear_s, 0, sizeof(shear_s));
    memset(thick_s, 0, sizeof(thick_s));
    if (ans_shear || ans_thick)
        for (int level = 0; level < 2; ++level) {
            const double zeta = level ? q : -q;
            for (int s = 0; s < 4; ++s) {
                if (ans_shear) {
                    point_t p;
                    double b[6][24];
                    evaluate(nodes, kShearSample[s][0], kShearSample[s][1], zeta, &p);
                    natural_b(&p, b);
                    for (int c = 0; c < 24; ++c) shear_s[level][s][c] = b[s < 2 ? 4 : 5][c];
                }
                if (ans_thick) {
                    point_t p;
                    double b[6][24];
                    evaluate(nodes, kCornerSample[s][0], kCornerSample[s][1], zeta, &p);
                    natural_b(&p, b);
                    for (int c = 0; c < 24; ++c) thick_s[level][s][c] = b[2][c];
                }
            }
        }

    for (int gp = 0; gp < 8; ++gp) {
        const double xi = (gp & 1) ? q : -q;
        const double eta = (gp & 2) ? q : -q;
        const double zta = (gp & 4) ? q : -q;
        const int level = (gp & 4) ? 1 : 0;
        point_t p;
        evaluate(nodes, xi, eta, zta, &p);
        double a[3][3];
        const double det = inv3(p.jac, a);
        if (!(det > 0.0)) {
            out[1506] = 0.0;
            return;
        }
        W[gp] = det;
        if (shape)
            for (int n = 0; n < 8; ++n)
                shape[gp][n] = 0.125 * (1.0 + xi * kXi[n]) * (1.0 + eta * kEta[n]) * (1.0 + zta * kZta[n]);
        double bn[6][24];
        natural_b(&p, bn);
        if (ans_shear) {
            const double wa = 0.5 * (1.0 - xi), wc = 0.5 * (1.0 + xi);
            const double wb = 0.5 * (1.0 - eta), wd = 0.5 * (1.0 + eta);
            for (int c = 0; c < 24; ++c) {
                bn[4][c] = wa * shear_s[level][0][c] + wc * shear_s[level][1][c];
                bn[5][c] = wb * shear_s[level][2][c] + wd * shear_s[level][3][c];
            }
        }
        if (ans_thick) {
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
                B[(gp * 6 + i) * 24 + c] = s;
            }
        if (!eas) {
            for (int i = 0; i < 6; ++i)
                for (int j = 0; j < 7; ++j) G[(gp * 6 + i) * 7 + j] = 0.0;
            continue;
        }
        double m[6][7];
        enhanced_m(xi, eta, zta, m);
        const double scale = det0 / det;
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 7; ++j) {
                double s = 0.0;
                for (int k = 0; k < 6; ++k) s += t0[i][k] * m[k][j];
                G[(gp * 6 + i) * 7 + j] = scale * s;
            }
    }
    if (eas) {
        for (int j = 0; j < 7; ++j) {
            double norm = 0.0;
            for (int gp = 0; gp < 8; ++gp)
                for (int i = 0; i < 6; ++i) norm += W[gp] * G[(gp * 6 + i) * 7 + j] * G[(gp * 6 + i) * 7 + j];
            if (!(norm > 0.0)) continue;
            const double inverse = 1.0 / sqrt(norm);
            for (int gp = 0; gp < 8; ++gp)
                for (int i = 0; i < 6; ++i) G[(gp * 6 + i) * 7 + j] *= inverse;
        }
    }
}

int or_shell_forms(const double rest[24], int formulation, double out[OR_FORMS_LEN]) {
    memset(out, 0, sizeof(double) * OR_FORMS_LEN);
    compute_forms(rest, formulation, out, NULL);
    return out[1506] != 0.0;
}

/* elementMass, solid_shell.cpp:655-663 */
void or_shell_mass(const double nodes[24], double density, double out[8]) {
    static double forms[OR_FORMS_LEN];
    double shape[8][8];
    for (int a = 0; a < 8; ++a) out[a] = 0.0;
    memset(forms, 0, sizeof(forms));
    compute_forms(nodes, 0, forms, shape);
    if (forms[1506] == 0.0) return;
    for (int gp = 0; gp < 8; ++gp)
        for (int a = 0; a < 8; ++a) out[a] += density * forms[1488 + gp] * shape[gp][a];
}

/* gaussVolumes, solid_shell.cpp:665-673 */
void or_shell_gauss_volumes(const double nodes[24], double out[8]) {
    static double forms[OR_FORMS_LEN];
    for (int gp = 0; gp < 8; ++gp) out[gp] = 0.0;
    memset(forms, 0, sizeof(forms));
    compute_forms(nodes, 0, forms, NULL);
    if (forms[1506] == 0.0) return;
    for (int gp = 0; gp < 8; ++gp) out[gp] = forms[1488 + gp];
}

/* elementSize, solid_shell.cpp:770-806 */
static void element_size(const double nodes[24], double *in_plane, double *thickness) {
    *in_plane = 0.0;
    *thickness = 0.0;
    double mid[4][3];
    for (int a = 0; a < 4; ++a)
        for (int i = 0; i < 3; ++i) mid[a][i] = 0.5 * (nodes[a * 3 + i] + nodes[(a + 4) * 3 + i]);
    double area = 0.0;
    for (int t = 0; t < 2; ++t) {
        const int b = t + 1, c = t + 2;
        double e1[3], e2[3];
        for (int i = 0; i < 3; ++i) {
            e1[i] = mid[b][i] - mid[0][i];
            e2[i] = mid[c][i] - mid[0][i];
        }
        const double cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                              e1[0] * e2[1] - e1[1] * e2[0]};
        area += 0.5 * sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    }
    if (!(area > 0.0)) return;
    static double forms[OR_FORMS_LEN];
    memset(forms, 0, sizeof(forms));
    compute_forms(nodes, 0, forms, NULL);
    if (forms[1506] == 0.0) return;
    double volume = 0.0;
    for (int gp = 0; gp < 8; ++gp) volume += forms[1488 + gp];
    *in_plane = sqrt(area);
    *thickness = volume / area;
}

/* initialisePlasticState, solid_shell.cpp:808-815, with
 * regularisedFailureStrain, plasticity.cpp:158-169 */
void or_shell_init_state(const double nodes[24], const double *mat, double state[OR_SHELL_STATE_LEN]) {
    for (int i = 0; i < OR_SHELL_STATE_LEN; ++i) state[i] = 0.0;
    double in_plane, thickness;
    element_size(nodes, &in_plane, &thickness);
    double share = 1.0;
    if (in_plane > 0.0 && thickness > 0.0) share = dmin(1.0, thickness / in_plane);
    state[127] = mat[9] + (mat[10] - mat[9]) * share;
}

/* solveSmall, solid_shell.cpp:432-457: dense Cholesky, n <= 7 */
static int solve_small(const double a[49], int n, double *rhs, int columns) {
    double l[49];
    for (int i = 0; i < 49; ++i) l[i] = 0.0;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j <= i; ++j) {
            double s = a[i * 7 + j];
            for (int k = 0; k < j; ++k) s -= l[i * 7 + k] * l[j * 7 + k];
            if (i == j) {
                if (!(s > 0.0)) return 0;
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
    return 1;
}

/* polarRotation, solid_shell.cpp:473-487 (to convergence, row-major) */
static void polar_rm(const double f[3][3], double r[3][3]) {
    memcpy(r, f, sizeof(double) * 9);
    for (int it = 0; it < 64; ++it) {
        double inv[3][3];
        if (inv3(r, inv) == 0.0) return;
        double worst = 0.0;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                const double next = 0.5 * (r[i][j] + inv[j][i]);
                worst = dmax(worst, fabs(next - r[i][j]));
                r[i][j] = next;
            }
        if (worst < 1e-16) return;
    }
}

/* elementRotation (cached), solid_shell.cpp:683-700 and rotationFrom :689 */
void or_shell_rotation(const double forms[OR_FORMS_LEN], const double current[24], double out[9]) {
    if (forms[1506] == 0.0) {
        for (int i = 0; i < 9; ++i) out[i] = (i % 4 == 0) ? 1.0 : 0.0;
        return;
    }
    point_t c;
    evaluate(current, 0.0, 0.0, 0.0, &c);
    double f[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += c.jac[i][k] * forms[1496 + k * 3 + j];
            f[i][j] = s;
        }
    double rot[3][3];
    polar_rm(f, rot);
    for (int col = 0; col < 3; ++col)
        for (int row = 0; row < 3; ++row) out[col * 3 + row] = rot[row][col];
}

/* elementPlasticUpdate (cached), solid_shell.cpp:826-1029: co-rotated displacement,
 * EAS Newton on r(alpha) = sum_gp w G^T sigma = 0 with the point law at every Gauss
 * point restarted from the step's start state, energy stopping rule, degraded retry,
 * commit, f = -R sum_gp w B^T sigma. */
int or_shell_plastic_update(const double forms[OR_FORMS_LEN], const double rest[24],
                            const double current[24], const double *mat,
                            double state[OR_SHELL_STATE_LEN], double force[24],
                            double stress[48], double info[7]) {
    double res[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 24; ++i) force[i] = 0.0;
    if (stress)
        for (int i = 0; i < 48; ++i) stress[i] = 0.0;
    if (forms[1506] == 0.0) {
        if (info) memcpy(info, res, sizeof(res));
        return 0;
    }
    const double *B = forms, *G = forms + 1152, *W = forms + 1488;
    double r[9];
    or_shell_rotation(forms, current, r);
    double u[24];
    for (int a = 0; a < 8; ++a)
        for (int i = 0; i < 3; ++i) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += r[i * 3 + k] * current[a * 3 + k];
            u[a * 3 + i] = s - rest[a * 3 + i];
        }
    int eas = (int)forms[1505];
    int degraded = 0;
    for (int gp = 0; gp < 8; ++gp) degraded = degraded || state[gp * OR_POINT_LEN + 14] != 0.0;
    if (degraded) eas = 0;
    double volume = 0.0;
    for (int gp = 0; gp < 8; ++gp) volume += W[gp];
    double start[8][OR_POINT_LEN];
    for (int gp = 0; gp < 8; ++gp) memcpy(start[gp], state + gp * OR_POINT_LEN, sizeof(start[gp]));
    double alpha[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int k = 0; k < eas; ++k) alpha[k] = state[120 + k];
    double trial[8][OR_POINT_LEN], incs[8][OR_INCR_LEN], gs[8][6], tangent[8][36];
    const double scale = mat[2] * volume;
    const double failure_strain = state[127];

    for (int attempt = 0; attempt < 2; ++attempt) {
        res[0] = 0.0;
        res[5] = 0.0;
        res[6] = 0.0;
        for (int iteration = 0;; ++iteration) {
            for (int gp = 0; gp < 8; ++gp) {
                double strain[6];
                for (int i = 0; i < 6; ++i) {
                    double s = 0.0;
                    for (int j = 0; j < 24; ++j) s += B[(gp * 6 + i) * 24 + j] * u[j];
                    for (int k = 0; k < eas; ++k) s += G[(gp * 6 + i) * 7 + k] * alpha[k];
                    strain[i] = s;
                }
                memcpy(trial[gp], start[gp], sizeof(trial[gp]));
                or_plastic_update(mat, failure_strain, strain, trial[gp], gs[gp], tangent[gp], incs[gp]);
            }
            res[1] = iteration + 1;
            if (eas == 0) {
                res[0] = 1.0;
                break;
            }
            double residual[7] = {0, 0, 0, 0, 0, 0, 0};
            for (int gp = 0; gp < 8; ++gp)
                for (int k = 0; k < eas; ++k) {
                    double s = 0.0;
                    for (int i = 0; i < 6; ++i) s += G[(gp * 6 + i) * 7 + k] * gs[gp][i];
                    residual[k] += W[gp] * s;
                }
            double norm = 0.0;
            for (int k = 0; k < eas; ++k) norm += residual[k] * residual[k];
            norm = sqrt(norm);
            res[5] = norm;
            if (norm <= 1e-12 * scale) {
                res[0] = 1.0;
                break;
            }
            if (iteration + 1 >= 40) break;
            double kaa[49];
            for (int i = 0; i < 49; ++i) kaa[i] = 0.0;
            for (int gp = 0; gp < 8; ++gp) {
                double cg[6][7];
                for (int i = 0; i < 6; ++i)
                    for (int k = 0; k < eas; ++k) {
                        double s = 0.0;
                        for (int mm = 0; mm < 6; ++mm) s += tangent[gp][i * 6 + mm] * G[(gp * 6 + mm) * 7 + k];
                        cg[i][k] = s;
                    }
                for (int p = 0; p < eas; ++p)
                    for (int q = 0; q < eas; ++q) {
                        double s = 0.0;
                        for (int i = 0; i < 6; ++i) s += G[(gp * 6 + i) * 7 + p] * cg[i][q];
                        kaa[p * 7 + q] += W[gp] * s;
                    }
            }
            double delta[7];
            for (int k = 0; k < eas; ++k) delta[k] = -residual[k];
            if (!solve_small(kaa, eas, delta, 1)) break;
            double work = 0.0;
            for (int k = 0; k < eas; ++k) work += delta[k] * residual[k];
            res[6] = fabs(work);
            if (res[6] <= 1e-16 * scale) {
                res[0] = 1.0;
                break;
            }
            for (int k = 0; k < eas; ++k) alpha[k] += delta[k];
        }
        int died = 0;
        for (int gp = 0; gp < 8; ++gp) died = died || trial[gp][14] != 0.0;
        if (!(died && eas > 0)) break;
        eas = 0;
        for (int k = 0; k < 7; ++k) alpha[k] = 0.0;
    }

    int failed = 0;
    for (int gp = 0; gp < 8; ++gp) {
        memcpy(state + gp * OR_POINT_LEN, trial[gp], sizeof(trial[gp]));
        res[4] += W[gp] * incs[gp][4];
        if (incs[gp][0] != 0.0) res[2] += 1.0;
        if (trial[gp][14] != 0.0) ++failed;
        if (stress)
            for (int i = 0; i < 6; ++i) stress[gp * 6 + i] = gs[gp][i];
    }
    res[3] = failed;
    for (int k = 0; k < 7; ++k) state[120 + k] = alpha[k];
    state[128] = failed == 8 ? 1.0 : 0.0;

    double internal[24];
    for (int j = 0; j < 24; ++j) internal[j] = 0.0;
    for (int gp = 0; gp < 8; ++gp)
        for (int j = 0; j < 24; ++j) {
            double s = 0.0;
            for (int i = 0; i < 6; ++i) s += B[(gp * 6 + i) * 24 + j] * gs[gp][i];
            internal[j] += W[gp] * s;
        }
    for (int a = 0; a < 8; ++a)
        for (int i = 0; i < 3; ++i) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += r[k * 3 + i] * internal[a * 3 + k];
            force[a * 3 + i] = -s;
        }
    if (info) memcpy(info, res, sizeof(res));
    return res[0] != 0.0;
}

/* isotropic C and computeBlocks (solid_shell.cpp:146-158, 377-429) and the static
 * condensation of elementStiffness (solid_shell.cpp:509-535) */
void or_shell_stiffness(const double nodes[24], double E, double nu, int formulation, double out[576]) {
    static double forms[OR_FORMS_LEN];
    for (int i = 0; i < 576; ++i) out[i] = 0.0;
    memset(forms, 0, sizeof(forms));
    compute_forms(nodes, formulation, forms, NULL);
    if (forms[1506] == 0.0) return;
    const double *B = forms, *G = forms + 1152, *W = forms + 1488;
    const int eas = (int)forms[1505];
    double c[6][6];
    {
        const double lambda = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
        const double mu = E / (2.0 * (1.0 + nu));
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 6; ++j) c[i][j] = 0.0;
        for (int i = 0; i < 3; ++i) {
            for (int j = 0; j < 3; ++j) c[i][j] = lambda;
            c[i][i] += 2.0 * mu;
            c[3 + i][3 + i] = mu;
        }
    }
    static double kuu[576];
    double kua[24 * 7], kaa[49];
    for (int i = 0; i < 576; ++i) kuu[i] = 0.0;
    for (int i = 0; i < 24 * 7; ++i) kua[i] = 0.0;
    for (int i = 0; i < 49; ++i) kaa[i] = 0.0;
    for (int gp = 0; gp < 8; ++gp) {
        const double w = W[gp];
        double cb[6][24];
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 24; ++j) {
                double s = 0.0;
                for (int k = 0; k < 6; ++k) s += c[i][k] * B[(gp * 6 + k) * 24 + j];
                cb[i][j] = s;
            }
        for (int i = 0; i < 24; ++i)
            for (int j = 0; j < 24; ++j) {
                double s = 0.0;
                for (int k = 0; k < 6; ++k) s += B[(gp * 6 + k) * 24 + i] * cb[k][j];
                kuu[i * 24 + j] += w * s;
            }
        if (eas == 0) continue;
        double cg[6][7];
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 7; ++j) {
                double s = 0.0;
                for (int k = 0; k < 6; ++k) s += c[i][k] * G[(gp * 6 + k) * 7 + j];
                cg[i][j] = s;
            }
        for (int i = 0; i < 24; ++i)
            for (int j = 0; j < 7; ++j) {
                double s = 0.0;
                for (int k = 0; k < 6; ++k) s += B[(gp * 6 + k) * 24 + i] * cg[k][j];
                kua[i * 7 + j] += w * s;
            }
        for (int i = 0; i < 7; ++i)
            for (int j = 0; j < 7; ++j) {
                double s = 0.0;
                for (int k = 0; k < 6; ++k) s += G[(gp * 6 + k) * 7 + i] * cg[k][j];
                kaa[i * 7 + j] += w * s;
            }
    }
    memcpy(out, kuu, sizeof(kuu));
    if (eas == 0) return;
    double x[7 * 24];
    for (int i = 0; i < eas; ++i)
        for (int j = 0; j < 24; ++j) x[i * 24 + j] = kua[j * 7 + i];
    if (!solve_small(kaa, eas, x, 24)) return;
    for (int i = 0; i < 24; ++i)
        for (int j = 0; j < 24; ++j) {
            double s = 0.0;
            for (int k = 0; k < eas; ++k) s += kua[i * 7 + k] * x[k * 24 + j];
            out[i * 24 + j] -= s;
        }
}

/* criticalTimestep (element), solid_shell.cpp:1088-1133 */
double or_shell_critical_dt(const double nodes[24], double E, double nu, double rho, int formulation,
                            double safety) {
    static double k[576];
    double m[8];
    or_shell_stiffness(nodes, E, nu, formulation, k);
    or_shell_mass(nodes, rho, m);
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
            for (int j = 0; j < 24; ++j) s += k[i * 24 + j] * (d[j] * v[j]);
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

void or_plate_sizes(int nx, int ny, int nz, size_t *nodes, size_t *elements) {
    *nodes = (size_t)(nx + 1) * (size_t)(ny + 1) * (size_t)(nz + 1);
    *elements = (size_t)nx * (size_t)ny * (size_t)nz;
}

/* makePlateMesh, solid_shell.cpp:1152-1185: thickness index fastest, then y, x;
 * mid-surface at z = 0. */
void or_plate_mesh(double lx, double ly, double thickness, int nx, int ny, int nz, double *position,
                   uint32_t *index) {
    const int sy = ny + 1, sz = nz + 1;
#define PAT(i, j, k) ((uint32_t)(((i) * sy + (j)) * sz + (k)))
    for (int i = 0; i <= nx; ++i)
        for (int j = 0; j <= ny; ++j)
            for (int k = 0; k <= nz; ++k) {
                double *p = &position[(size_t)PAT(i, j, k) * 3];
                p[0] = lx * (double)i / nx;
                p[1] = ly * (double)j / ny;
                p[2] = -0.5 * thickness + thickness * (double)k / nz;
            }
    size_t e = 0;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                const uint32_t v[8] = {PAT(i, j, k),         PAT(i + 1, j, k),         PAT(i + 1, j + 1, k),
                                       PAT(i, j + 1, k),     PAT(i, j, k + 1),         PAT(i + 1, j, k + 1),
                                       PAT(i + 1, j + 1, k + 1), PAT(i, j + 1, k + 1)};
                memcpy(&index[e * 8], v, sizeof(v));
                ++e;
            }
#undef PAT
}

/* uniformPressureLoad, solid_shell.cpp:1505-1553, for meshes where every element's
 * +zeta face is on the boundary (one element through the thickness): 2x2 Gauss
 * consistent loads on the top face, pushing along -(x_s x x_t). */
void or_plate_pressure_load(const double *position, const uint32_t *index, size_t nodes, size_t elements,
                            double pressure, double *load) {
    static const double corner[4][2] = {{-1, -1}, {+1, -1}, {+1, +1}, {-1, +1}};
    for (size_t i = 0; i < nodes * 3; ++i) load[i] = 0.0;
    const double q = 1.0 / sqrt(3.0);
    for (size_t e = 0; e < elements; ++e) {
        uint32_t n[4];
        for (int i = 0; i < 4; ++i) n[i] = index[e * 8 + 4 + i];
        for (int gs = 0; gs < 2; ++gs)
            for (int gt = 0; gt < 2; ++gt) {
                const double s = gs ? q : -q, t = gt ? q : -q;
                double shape[4], ds[4], dt[4];
                for (int c = 0; c < 4; ++c) {
                    shape[c] = 0.25 * (1.0 + s * corner[c][0]) * (1.0 + t * corner[c][1]);
                    ds[c] = 0.25 * corner[c][0] * (1.0 + t * corner[c][1]);
                    dt[c] = 0.25 * corner[c][1] * (1.0 + s * corner[c][0]);
                }
                double xs[3] = {0, 0, 0}, xt[3] = {0, 0, 0};
                for (int c = 0; c < 4; ++c)
                    for (int i = 0; i < 3; ++i) {
                        xs[i] += ds[c] * position[(size_t)n[c] * 3 + i];
                        xt[i] += dt[c] * position[(size_t)n[c] * 3 + i];
                    }
                const double area[3] = {xs[1] * xt[2] - xs[2] * xt[1], xs[2] * xt[0] - xs[0] * xt[2],
                                        xs[0] * xt[1] - xs[1] * xt[0]};
                for (int c = 0; c < 4; ++c)
                    for (int i = 0; i < 3; ++i) load[(size_t)n[c] * 3 + i] -= pressure * shape[c] * area[i];
            }
    }
}

/* Solver set-up, zone.cpp:698-754 */
void or_shell_setup(or_shell *m, const double *mat, double density) {
    for (size_t n = 0; n < m->nodes; ++n) m->mass[n] = 0.0;
    for (size_t e = 0; e < m->elements; ++e) {
        double nodes[24];
        for (int a = 0; a < 8; ++a)
            for (int i = 0; i < 3; ++i) nodes[a * 3 + i] = m->rest[(size_t)m->index[e * 8 + a] * 3 + i];
        or_shell_forms(nodes, 2, m->forms + e * OR_FORMS_LEN);
        double lumped[8];
        or_shell_mass(nodes, density, lumped);
        for (int a = 0; a < 8; ++a) m->mass[m->index[e * 8 + a]] += lumped[a];
        or_shell_init_state(nodes, mat, m->state + e * OR_SHELL_STATE_LEN);
        or_shell_gauss_volumes(nodes, m->gauss_volume + e * 8);
    }
    build_csr(m->nodes, m->elements, 8, m->index, m->adj_offset, m->adj_entry);
}

/* Solver::step for a patch with no punch and no driven edge, with an external
 * nodal load: zone.cpp:928-989, 1094-1121, 1200-1202. */
/* The uniaxial return of a fibre (constraint.cpp:39-95): backward Euler on the flow
   rule, isotropic hardening only, a Newton solve of the consistency condition (32
   iterations, 1e-13 relative), then the damage increment with the bar's closed-form
   triaxiality +-1/3 (constraint.cpp:102-109).  st: plastic strain, eq. plastic
   strain, damage, failed. */
static double fiber_return(const double *mat, double failure_strain, double strain, double *st,
                           double *dissipation_per_volume) {
    *dissipation_per_volume = 0.0;
    if (st[3] != 0.0) return 0.0;
    const double youngs = mat[0];
    const double trial = youngs * (strain - st[0]);
    const double yield = flow_stress(mat, st[1]);
    if (fabs(trial) <= yield) return trial;
    const double slope0 = flow_slope(mat, st[1]);
    double increment = (fabs(trial) - yield) / (youngs + slope0);
    for (int it = 0; it < 32; ++it) {
        const double residual = fabs(trial) - youngs * increment - flow_stress(mat, st[1] + increment);
        if (fabs(residual) <= 1e-13 * (yield + fabs(trial))) break;
        const double slope = youngs + flow_slope(mat, st[1] + increment);
        if (!(slope > 0)) break;
        increment += residual / slope;
        if (increment < 0) increment = 0;
    }
    const double direction = trial >= 0 ? 1.0 : -1.0;
    const double stress = trial - direction * youngs * increment;
    st[0] += direction * increment;
    st[1] += increment;
    *dissipation_per_volume = fabs(stress) * increment;
    const double eta = stress == 0.0 ? 0.0 : (stress > 0.0 ? 1.0 : -1.0) / 3.0;
    const double critical = failure_strain * triax_factor(mat, eta);
    if (critical > 0.0 && isfinite(critical)) st[2] += increment / critical;
    if (st[2] >= 1.0) {
        st[2] = 1.0;
        st[3] = 1.0;
        return 0.0;
    }
    return stress;
}

/* fiberForces (constraint.cpp:198-258): every fibre's co-rotational axial force, added
   into `force` through its ties in fibre order.  Returns the plastic dissipation of
   the increment; the recoverable strain energy goes to m->fiber_energy. */
static double fiber_forces(or_shell *m, const double *mat, double *force) {
    double dissipation = 0.0, energy = 0.0;
    const double youngs = mat[0];
    for (size_t i = 0; i < m->fibers; ++i) {
        const double rest_length = m->fiber_length[i], area = m->fiber_area[i];
        if (!(rest_length > 0) || !(area > 0)) continue;
        const uint32_t *tie = m->fiber_tie + i * 4;
        const double *w = m->fiber_weight + i * 2;
        double end[2][3];
        for (int e = 0; e < 2; ++e)
            for (int k = 0; k < 3; ++k)
                end[e][k] = m->position[(size_t)tie[2 * e] * 3 + k] * (1.0 - w[e]) +
                            m->position[(size_t)tie[2 * e + 1] * 3 + k] * w[e];
        double span[3];
        for (int k = 0; k < 3; ++k) span[k] = end[1][k] - end[0][k];
        const double l = sqrt(span[0] * span[0] + span[1] * span[1] + span[2] * span[2]);
        if (!(l > 0)) continue;
        double axis[3];
        for (int k = 0; k < 3; ++k) axis[k] = span[k] / l;
        const double strain = (l - rest_length) / rest_length;
        double dpv = 0.0;
        const double stress = fiber_return(mat, m->fiber_fail[i], strain, m->fiber_state + i * 4, &dpv);
        dissipation += dpv * area * rest_length;
        const double axial = stress * area;
        for (int e = 0; e < 2; ++e) {
            const double sign_axial = e == 0 ? axial : -axial;
            const size_t bottom = (size_t)tie[2 * e] * 3, top = (size_t)tie[2 * e + 1] * 3;
            for (int k = 0; k < 3; ++k) {
                const double f = axis[k] * sign_axial;
                force[bottom + k] += (1.0 - w[e]) * f;
                force[top + k] += w[e] * f;
            }
        }
        energy += 0.5 * stress * stress / youngs * area * rest_length;
    }
    m->fiber_energy = energy;
    return dissipation;
}

/* The element part of one shell step for element e (zone.cpp:964-973): its forces,
 * stresses and state, and its dissipation into diss[e] (0 for a torn element). */
static void shell_element(or_shell *m, const double *mat, size_t e, double *diss) {
    double rest[24], current[24];
    for (int a = 0; a < 8; ++a)
        for (int i = 0; i < 3; ++i) {
            rest[a * 3 + i] = m->rest[(size_t)m->index[e * 8 + a] * 3 + i];
            current[a * 3 + i] = m->position[(size_t)m->index[e * 8 + a] * 3 + i];
        }
    double *st = m->state + e * OR_SHELL_STATE_LEN;
    double *out = m->element_force + e * 24;
    double *stress = m->stress + e * 48;
    diss[e] = 0.0;
    if (st[128] != 0.0) {
        for (int i = 0; i < 24; ++i) out[i] = 0.0;
        for (int i = 0; i < 48; ++i) stress[i] = 0.0;
        return;
    }
    double info[7];
    or_shell_plastic_update(m->forms + e * OR_FORMS_LEN, rest, current, mat, st, out, stress, info);
    diss[e] = info[4];
}

typedef struct {
    or_shell *m;
    const double *mat;
    size_t begin, end;
    double *diss;
} shell_range;

static void *shell_range_run(void *arg) {
    const shell_range *r = (const shell_range *)arg;
    for (size_t e = r->begin; e < r->end; ++e) shell_element(r->m, r->mat, e, r->diss);
    return NULL;
}

/* Steps of the composed shell step: the element loop (shell_element), over `threads`
 * host threads when threads > 1, then the gather and the node update.  The element
 * dissipations are summed in element order, skipping torn elements as the serial loop
 * does, so every thread count gives the same bits. */
static void shell_steps(or_shell *m, const double *mat, const or_shell_params *p, int steps, int threads) {
    /* the velocity each driven-edge DOF would have taken had nothing held it */
    double *edge_free = m->prescribed ? (double *)calloc(m->nodes * 3, sizeof(double)) : NULL;
    double *gathered = (double *)malloc(m->nodes * 3 * sizeof(double));
    double *diss = (double *)malloc((m->elements + 1) * sizeof(double));
    unsigned char *torn = (unsigned char *)malloc(m->elements + 1);
    if (!gathered || !diss || !torn) abort();
    for (int s = 0; s < steps && !m->arrested; ++s) {
        const double time = (double)(m->step + 1) * p->dt;
        const double lf = p->rise_time > 0 ? dmin(time / p->rise_time, 1.0) : 1.0;
        for (size_t e = 0; e < m->elements; ++e) torn[e] = m->state[e * OR_SHELL_STATE_LEN + 128] != 0.0;
        if (threads > 1) {
            pthread_t tid[OR_MAX_THREADS];
            shell_range job[OR_MAX_THREADS];
            const int n = threads < OR_MAX_THREADS ? threads : OR_MAX_THREADS;
            for (int k = 0; k < n; ++k) {
                job[k] = (shell_range){m, mat, m->elements * k / n, m->elements * (k + 1) / n, diss};
                if (pthread_create(&tid[k], NULL, shell_range_run, &job[k])) abort();
            }
            for (int k = 0; k < n; ++k) pthread_join(tid[k], NULL);
        } else {
            for (size_t e = 0; e < m->elements; ++e) shell_element(m, mat, e, diss);
        }
        double dissipation = 0.0;
        for (size_t e = 0; e < m->elements; ++e)
            if (!torn[e]) dissipation += diss[e];
        /* the gather (zone.cpp:976-989), then the stiffeners' forces through their ties,
           in fibre order (zone.cpp:990-1002) */
        for (size_t node = 0; node < m->nodes; ++node) {
            double sum[3] = {0, 0, 0};
            for (uint32_t k = m->adj_offset[node]; k < m->adj_offset[node + 1]; ++k) {
                const uint32_t entry = m->adj_entry[k];
                const double *f = &m->element_force[(size_t)(entry / 8) * 24 + (entry % 8) * 3];
                sum[0] += f[0];
                sum[1] += f[1];
                sum[2] += f[2];
            }
            for (int k = 0; k < 3; ++k) gathered[node * 3 + (size_t)k] = sum[k];
        }
        if (m->fibers) dissipation += fiber_forces(m, mat, gathered);
        /* force -> velocity (zone.cpp:1094-1111); the kinetic energy before the damping
           and the damping's loss (zone.cpp:1113-1121) */
        double work = 0.0, before = 0.0;
        for (size_t node = 0; node < m->nodes; ++node) {
            double ext[3];
            for (int k = 0; k < 3; ++k) {
                const size_t d = node * 3 + (size_t)k;
                ext[k] = m->fext ? lf * m->fext[d] : 0.0;
                const double force = gathered[d] + ext[k];
                if (m->pinned[d]) {
                    if (edge_free && m->prescribed[d] != 0.0) {
                        double free_velocity = m->velocity[d];
                        if (m->mass[node] > 0) free_velocity += force / m->mass[node] * p->dt;
                        edge_free[d] = free_velocity;
                    }
                    m->velocity[d] = 0.0;
                    continue;
                }
                if (m->mass[node] > 0) m->velocity[d] += force / m->mass[node] * p->dt;
            }
            const double *v = &m->velocity[node * 3];
            before += 0.5 * m->mass[node] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            for (int k = 0; k < 3; ++k) {
                const size_t d = node * 3 + (size_t)k;
                if (m->pinned[d]) continue;
                m->velocity[d] *= p->damping;
                work += ext[k] * m->velocity[d] * p->dt;
            }
        }
        if (p->damping != 1.0) m->account[0] += before * (1.0 - p->damping * p->damping);
        /* the driven edge, after the damping and before the punch (zone.cpp:1123-1145):
           the velocity that lands the DOF on its drive this step; the boundary's work is
           what that velocity costs over the free one */
        if (edge_free) {
            double fraction = 1.0;
            if (m->edge_ramp > 0) {
                /* the time at the step's end, as the running sum the solver keeps */
                const double r = dmin(1.0, dmax(0.0, (m->account[3] + p->dt) / m->edge_ramp));
                fraction = r * r * (3.0 - 2.0 * r);
            }
            for (size_t d = 0; d < m->nodes * 3; ++d) {
                if (!m->pinned[d] || m->prescribed[d] == 0.0) continue;
                const size_t node = d / 3;
                const double base = m->meshed ? m->meshed[d] : m->rest[d];
                const double target = (base + m->prescribed[d] * fraction - m->position[d]) / p->dt;
                m->account[1] += m->mass[node] * (target - edge_free[d]) * target;
                m->velocity[d] = target;
            }
        }
        /* the punch, after the edge and before the positions (zone.cpp:1147-1198): each
           gripped node moves at -speed along the axis; the impulse that takes is the
           resisting force.  Prescribed: the speed ramps from the time at the start of the
           step.  Inertial: the grip is a perfectly inelastic collision of the striking
           body with the gripped nodes, momentum along the axis conserved. */
        double speed = 0.0;
        if (m->driven) {
            const double t0 = m->account[3];  /* the time at the step's start (a running sum) */
            speed = p->punch_speed;
            if (p->punch_ramp > 0 && t0 < p->punch_ramp) speed = p->punch_speed * (t0 / p->punch_ramp);
            if (m->punch_mass > 0) {
                double node_momentum = 0.0, driven_mass = 0.0;
                for (size_t node = 0; node < m->nodes; ++node) {
                    if (!m->driven[node]) continue;
                    const double *v = &m->velocity[node * 3];
                    node_momentum -= m->mass[node] * (v[0] * m->axis[0] + v[1] * m->axis[1] + v[2] * m->axis[2]);
                    driven_mass += m->mass[node];
                }
                m->punch_velocity = (m->punch_mass * m->punch_velocity + node_momentum) / (m->punch_mass + driven_mass);
                speed = m->punch_velocity;
            }
            double impulse = 0.0;
            for (size_t node = 0; node < m->nodes; ++node) {
                if (!m->driven[node]) continue;
                double *v = &m->velocity[node * 3];
                const double along = v[0] * m->axis[0] + v[1] * m->axis[1] + v[2] * m->axis[2];
                const double change = -speed - along;
                for (int k = 0; k < 3; ++k) v[k] += change * m->axis[k];
                impulse += m->mass[node] * change;
            }
            const double force = -impulse / p->dt;
            m->energy[4] += force * speed * p->dt;
        }
        for (size_t d = 0; d < m->nodes * 3; ++d) m->position[d] += m->velocity[d] * p->dt;
        m->account[2] += speed * p->dt;
        m->account[3] += p->dt;
        m->energy[0] += work;
        m->energy[1] += dissipation;
        ++m->step;
        /* the striking body has spent what it arrived with (zone.cpp:1225-1230) */
        if (m->driven && m->punch_mass > 0 && !(m->punch_velocity > 0)) m->arrested = 1;
    }
    free(edge_free);
    free(gathered);
    free(diss);
    free(torn);
}

/* Steps of the composed shell step (zone.cpp:1086-1252), serial. */
void or_shell_step(or_shell *m, const double *mat, const or_shell_params *p, int steps) {
    shell_steps(m, mat, p, steps, 1);
}

/* The same steps with the element loop over `threads` host threads: bit-identical to
 * or_shell_step, for the larger panels the GPU checks use. */
void or_shell_step_threads(or_shell *m, const double *mat, const or_shell_params *p, int steps, int threads) {
    shell_steps(m, mat, p, steps, threads);
}

/* accumulateEnergy, zone.cpp:1014-1044 */
void or_shell_energy(or_shell *m, const double *mat) {
    const double mu = mat[0] / (2.0 * (1.0 + mat[1]));
    const double bulk = mat[0] / (3.0 * (1.0 - 2.0 * mat[1]));
    double kinetic = 0;
    for (size_t node = 0; node < m->nodes; ++node) {
        const double *v = &m->velocity[node * 3];
        kinetic += 0.5 * m->mass[node] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    }
    double strain = 0;
    for (size_t e = 0; e < m->elements; ++e)
        for (int gp = 0; gp < 8; ++gp) {
            const double *s = &m->stress[e * 48 + (size_t)gp * 6];
            const double pressure = (s[0] + s[1] + s[2]) / 3.0;
            double density = 0;
            for (int i = 0; i < 3; ++i) density += 0.5 * s[i] * ((s[i] - pressure) / (2.0 * mu) + pressure / (3.0 * bulk));
            for (int i = 3; i < 6; ++i) density += 0.5 * s[i] * (s[i] / mu);
            strain += m->gauss_volume[e * 8 + gp] * density;
        }
    m->energy[2] = strain;
    m->energy[3] = kinetic;
}
