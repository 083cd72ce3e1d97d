// ref_shim.cpp -- C entry points over the reference's own compiled FEM code.
//
// TEST INFRASTRUCTURE ONLY: this file is compiled, together with the reference's
// unmodified sources (engine/sim/{fem,plasticity,solid_shell,zone,constraint,
// scantlings}.cpp, engine/core/{geometry,jobs}.cpp), into oracle/_ref/libshipsim_ref.so
// by oracle/Makefile.  It is the "reference" implementation behind the C interface of
// femoracle.h: every `ref_*` function here has an `or_*` twin in femoracle.c, and the
// tests check the pair against each other.
//
// Where the reference has the function, the shim only marshals arrays and calls it.
// Where a workload composes something the reference does not have in one piece
// (the J2 tet, the pressure-loaded shell step), the composition is written here on
// top of the reference's functions, and says which ones.
#include "engine/core/jobs.hpp"
#include "engine/sim/constraint.hpp"
#include "engine/sim/fem.hpp"
#include "engine/sim/plasticity.hpp"
#include "engine/sim/scantlings.hpp"
#include "engine/sim/solid_shell.hpp"
#include "engine/sim/zone.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "femoracle.h"

namespace pl = sim::plasticity;
namespace ss = sim::solidshell;
namespace fem = sim::fem;

namespace {

pl::Material toMaterial(const double* m) {
    pl::Material out;
    out.youngsModulus = m[0];
    out.poissonRatio = m[1];
    out.flow.yieldStrength = m[2];
    out.flow.hardeningModulus = m[3];
    out.flow.kinematicModulus = m[4];
    out.flow.kind = m[5] != 0.0 ? pl::Hardening::Swift : pl::Hardening::Linear;
    out.flow.strengthCoefficient = m[6];
    out.flow.referenceStrain = m[7];
    out.flow.hardeningExponent = m[8];
    out.failure.uniformStrain = m[9];
    out.failure.fractureStrain = m[10];
    out.failure.triaxialitySensitivity = m[11];
    out.failure.referenceTriaxiality = m[12];
    out.failure.cutoffTriaxiality = m[13];
    return out;
}

void pointIn(const double* s, pl::State& st) {
    for (int i = 0; i < 6; ++i) {
        st.plasticStrain[i] = s[i];
        st.backStress[i] = s[6 + i];
    }
    st.equivalentPlasticStrain = s[12];
    st.damage = s[13];
    st.failed = s[14] != 0.0;
}

void pointOut(const pl::State& st, double* s) {
    for (int i = 0; i < 6; ++i) {
        s[i] = st.plasticStrain[i];
        s[6 + i] = st.backStress[i];
    }
    s[12] = st.equivalentPlasticStrain;
    s[13] = st.damage;
    s[14] = st.failed ? 1.0 : 0.0;
}

void shellStateIn(const double* s, ss::ElementPlasticState& st) {
    for (int gp = 0; gp < ss::kGauss; ++gp) pointIn(s + gp * OR_POINT_LEN, st.point[gp]);
    for (int k = 0; k < ss::kEas; ++k) st.enhanced[k] = s[120 + k];
    st.failureStrain = s[127];
    st.torn = s[128] != 0.0;
}

void shellStateOut(const ss::ElementPlasticState& st, double* s) {
    for (int gp = 0; gp < ss::kGauss; ++gp) pointOut(st.point[gp], s + gp * OR_POINT_LEN);
    for (int k = 0; k < ss::kEas; ++k) s[120 + k] = st.enhanced[k];
    s[127] = st.failureStrain;
    s[128] = st.torn ? 1.0 : 0.0;
}

void formsIn(const double* f, ss::RestForms& out) {
    std::memcpy(out.b, f, sizeof(out.b));
    std::memcpy(out.g, f + 1152, sizeof(out.g));
    std::memcpy(out.weight, f + 1488, sizeof(out.weight));
    std::memcpy(out.restJacobianInverse, f + 1496, sizeof(out.restJacobianInverse));
    out.easCount = static_cast<int>(f[1505]);
    out.ok = f[1506] != 0.0;
}

void formsOut(const ss::RestForms& in, double* f) {
    std::memcpy(f, in.b, sizeof(in.b));
    std::memcpy(f + 1152, in.g, sizeof(in.g));
    std::memcpy(f + 1488, in.weight, sizeof(in.weight));
    std::memcpy(f + 1496, in.restJacobianInverse, sizeof(in.restJacobianInverse));
    f[1505] = in.easCount;
    f[1506] = in.ok ? 1.0 : 0.0;
}

ss::Formulation formOf(int f) {
    return f == 0 ? ss::Formulation::Displacement
                  : (f == 1 ? ss::Formulation::AssumedNaturalStrain : ss::Formulation::SolidShell);
}

fem::TetMesh toTetMesh(const or_tet32* m) {
    fem::TetMesh t;
    t.position.assign(m->position, m->position + m->nodes * 3);
    t.velocity.assign(m->velocity, m->velocity + m->nodes * 3);
    t.mass.assign(m->mass, m->mass + m->nodes);
    t.fixed.assign(m->fixed, m->fixed + m->nodes);
    t.index.assign(m->index, m->index + m->tets * 4);
    t.restInv.assign(m->rest_inv, m->rest_inv + m->tets * 9);
    t.restVolume.assign(m->rest_volume, m->rest_volume + m->tets);
    t.tetForce.assign(m->tet_force, m->tet_force + m->tets * 12);
    t.adjacencyOffset.assign(m->adj_offset, m->adj_offset + m->nodes + 1);
    t.adjacencyEntry.assign(m->adj_entry, m->adj_entry + m->tets * 4);
    return t;
}

void fromTetMesh(const fem::TetMesh& t, or_tet32* m) {
    std::copy(t.position.begin(), t.position.end(), m->position);
    std::copy(t.velocity.begin(), t.velocity.end(), m->velocity);
    std::copy(t.mass.begin(), t.mass.end(), m->mass);
    std::copy(t.fixed.begin(), t.fixed.end(), m->fixed);
    std::copy(t.restInv.begin(), t.restInv.end(), m->rest_inv);
    std::copy(t.restVolume.begin(), t.restVolume.end(), m->rest_volume);
    std::copy(t.tetForce.begin(), t.tetForce.end(), m->tet_force);
    std::copy(t.adjacencyOffset.begin(), t.adjacencyOffset.end(), m->adj_offset);
    std::copy(t.adjacencyEntry.begin(), t.adjacencyEntry.end(), m->adj_entry);
}

// --- the J2 tet in double: fem.cpp's kinematics restated, the point law called ---

struct M3d {
    double m[9];  // column-major, as fem.cpp's M3
    double& operator()(int r, int c) { return m[c * 3 + r]; }
    double operator()(int r, int c) const { return m[c * 3 + r]; }
};

M3d mul(const M3d& a, const M3d& b) {
    M3d r{};
    for (int c = 0; c < 3; ++c)
        for (int i = 0; i < 3; ++i) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += a(i, k) * b(k, c);
            r(i, c) = s;
        }
    return r;
}

M3d tr(const M3d& a) {
    M3d r{};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r(i, j) = a(j, i);
    return r;
}

double det(const M3d& a) {
    return a(0, 0) * (a(1, 1) * a(2, 2) - a(1, 2) * a(2, 1)) -
           a(0, 1) * (a(1, 0) * a(2, 2) - a(1, 2) * a(2, 0)) +
           a(0, 2) * (a(1, 0) * a(2, 1) - a(1, 1) * a(2, 0));
}

M3d inv(const M3d& a) {
    const double d = det(a);
    const double id = std::abs(d) > 1e-300 ? 1.0 / d : 0.0;
    M3d r{};
    r(0, 0) = (a(1, 1) * a(2, 2) - a(1, 2) * a(2, 1)) * id;
    r(0, 1) = (a(0, 2) * a(2, 1) - a(0, 1) * a(2, 2)) * id;
    r(0, 2) = (a(0, 1) * a(1, 2) - a(0, 2) * a(1, 1)) * id;
    r(1, 0) = (a(1, 2) * a(2, 0) - a(1, 0) * a(2, 2)) * id;
    r(1, 1) = (a(0, 0) * a(2, 2) - a(0, 2) * a(2, 0)) * id;
    r(1, 2) = (a(0, 2) * a(1, 0) - a(0, 0) * a(1, 2)) * id;
    r(2, 0) = (a(1, 0) * a(2, 1) - a(1, 1) * a(2, 0)) * id;
    r(2, 1) = (a(0, 1) * a(2, 0) - a(0, 0) * a(2, 1)) * id;
    r(2, 2) = (a(0, 0) * a(1, 1) - a(0, 1) * a(1, 0)) * id;
    return r;
}

// Higham iteration; fixed count (fem.cpp:62) or to convergence (solid_shell.cpp:473).
M3d polar(const M3d& f, int fixed) {
    M3d r = f;
    const int limit = fixed > 0 ? fixed : 64;
    for (int it = 0; it < limit; ++it) {
        if (fixed <= 0 && det(r) == 0.0) return r;
        const M3d rit = tr(inv(r));
        double worst = 0;
        for (int k = 0; k < 9; ++k) {
            const double next = 0.5 * (r.m[k] + rit.m[k]);
            worst = std::max(worst, std::abs(next - r.m[k]));
            r.m[k] = next;
        }
        if (fixed <= 0 && worst < 1e-16) return r;
    }
    return r;
}

}  // namespace

extern "C" {

int ref_plastic_update(const double* mat, double failure_strain, const double strain[6],
                       double state[OR_POINT_LEN], double stress[6], double* tangent,
                       double incr[OR_INCR_LEN]) {
    const pl::Material material = toMaterial(mat);
    pl::State st;
    pointIn(state, st);
    const pl::Increment inc = pl::update(material, failure_strain, strain, st, stress, tangent);
    pointOut(st, state);
    if (incr) {
        incr[0] = inc.yielded;
        incr[1] = inc.failedNow;
        incr[2] = inc.plasticMultiplier;
        incr[3] = inc.equivalentPlasticStrainIncrement;
        incr[4] = inc.dissipation;
        incr[5] = inc.plasticWork;
        incr[6] = inc.vonMises;
        incr[7] = inc.triaxiality;
        incr[8] = inc.iterations;
    }
    return inc.yielded ? 1 : 0;
}

void ref_box_tet_sizes(int nx, int ny, int nz, size_t* nodes, size_t* tets) {
    *nodes = static_cast<size_t>(nx + 1) * (ny + 1) * (nz + 1);
    *tets = static_cast<size_t>(nx) * ny * nz * 6;
}

void ref_box_tet_mesh(float lx, float ly, float lz, int nx, int ny, int nz, float* position,
                      uint32_t* index) {
    const fem::TetMesh t = fem::makeBoxTetMesh(lx, ly, lz, nx, ny, nz);
    std::copy(t.position.begin(), t.position.end(), position);
    std::copy(t.index.begin(), t.index.end(), index);
}

void ref_tet32_rest_state(or_tet32* m, float E, float nu, float rho) {
    fem::TetMesh t;
    t.position.assign(m->position, m->position + m->nodes * 3);
    t.index.assign(m->index, m->index + m->tets * 4);
    t.fixed.assign(m->fixed, m->fixed + m->nodes);
    fem::Material mat;
    mat.youngsModulus = E;
    mat.poissonRatio = nu;
    mat.density = rho;
    t.computeRestState(mat);
    fromTetMesh(t, m);
}

void ref_tet32_forces(const or_tet32* m, size_t t, float lambda, float mu, float out[12]) {
    const fem::TetMesh mesh = toTetMesh(m);
    fem::tetForces(mesh, t, lambda, mu, out);
}

void ref_tet32_step(or_tet32* m, float E, float nu, float rho, float dt, float gravity,
                    float damping, int steps) {
    fem::TetMesh t = toTetMesh(m);
    fem::Material mat;
    mat.youngsModulus = E;
    mat.poissonRatio = nu;
    mat.density = rho;
    for (int s = 0; s < steps; ++s) fem::stepCpu(t, mat, dt, gravity, damping);
    fromTetMesh(t, m);
}

float ref_tet32_critical_dt(const or_tet32* m, float E, float nu, float rho, float safety) {
    const fem::TetMesh t = toTetMesh(m);
    fem::Material mat;
    mat.youngsModulus = E;
    mat.poissonRatio = nu;
    mat.density = rho;
    return fem::criticalTimestep(t, mat, safety);
}

// O-tet64 rest state: fem.cpp:119-158 restated in double (computeRestState).
void ref_tet64_rest_state(or_tet64* m, double rho) {
    for (size_t n = 0; n < m->nodes; ++n) m->mass[n] = 0.0;
    for (size_t t = 0; t < m->tets; ++t) {
        const uint32_t* idx = &m->index[t * 4];
        M3d dm{};
        for (int c = 0; c < 3; ++c)
            for (int a = 0; a < 3; ++a)
                dm(a, c) = m->position[idx[c + 1] * 3 + a] - m->position[idx[0] * 3 + a];
        const double volume = det(dm) / 6.0;
        m->rest_volume[t] = std::abs(volume);
        const M3d i = inv(dm);
        for (int k = 0; k < 9; ++k) m->rest_inv[t * 9 + k] = i.m[k];
        const double quarter = rho * m->rest_volume[t] * 0.25;
        for (int c = 0; c < 4; ++c) m->mass[idx[c]] += quarter;
    }
    std::vector<uint32_t> off(m->nodes + 1, 0u);
    for (size_t t = 0; t < m->tets; ++t)
        for (int c = 0; c < 4; ++c) ++off[m->index[t * 4 + c] + 1];
    for (size_t n = 0; n < m->nodes; ++n) off[n + 1] += off[n];
    std::copy(off.begin(), off.end(), m->adj_offset);
    std::vector<uint32_t> cursor(off.begin(), off.end() - 1);
    for (size_t t = 0; t < m->tets; ++t)
        for (uint32_t c = 0; c < 4; ++c)
            m->adj_entry[cursor[m->index[t * 4 + c]]++] = static_cast<uint32_t>(t) * 4 + c;
}

// O-tet64 step: tetForces (fem.cpp:73-117) in double with plasticity::update at the
// single point, then the node loop of fem.cpp:196-214 with the external force added
// after the CSR gather.
void ref_tet64_step(or_tet64* m, const or_tet64_params* p, int steps) {
    pl::Material mat;
    mat.youngsModulus = p->E;
    mat.poissonRatio = p->nu;
    mat.flow = pl::linearHardening(p->yield, p->hardening);
    const double mu = mat.shearModulus(), bulk = mat.bulkModulus();
    for (int s = 0; s < steps; ++s) {
        const double lf =
            p->ramp_steps > 0
                ? std::min(static_cast<double>(m->step + 1) / static_cast<double>(p->ramp_steps), 1.0)
                : 1.0;
        double strainEnergy = 0.0, dissipation = 0.0;
        for (size_t t = 0; t < m->tets; ++t) {
            const uint32_t* idx = &m->index[t * 4];
            const double* x = m->position;
            M3d ds{};
            for (int c = 0; c < 3; ++c)
                for (int a = 0; a < 3; ++a) ds(a, c) = x[idx[c + 1] * 3 + a] - x[idx[0] * 3 + a];
            M3d dmInv{};
            for (int k = 0; k < 9; ++k) dmInv.m[k] = m->rest_inv[t * 9 + k];
            const M3d f = mul(ds, dmInv);
            const M3d r = polar(f, p->polar_fixed);
            const M3d sm = mul(tr(r), f);
            double strain[6];
            strain[0] = 0.5 * (sm(0, 0) + sm(0, 0)) - 1.0;
            strain[1] = 0.5 * (sm(1, 1) + sm(1, 1)) - 1.0;
            strain[2] = 0.5 * (sm(2, 2) + sm(2, 2)) - 1.0;
            strain[3] = 2.0 * (0.5 * (sm(0, 1) + sm(1, 0)));
            strain[4] = 2.0 * (0.5 * (sm(1, 2) + sm(2, 1)));
            strain[5] = 2.0 * (0.5 * (sm(2, 0) + sm(0, 2)));
            pl::State st;
            const double* ps = &m->plastic[t * 7];
            for (int i = 0; i < 6; ++i) st.plasticStrain[i] = ps[i];
            st.equivalentPlasticStrain = ps[6];
            double sv[6];
            const pl::Increment inc = pl::update(mat, pl::kNeverFails, strain, st, sv);
            double* pw = &m->plastic[t * 7];
            for (int i = 0; i < 6; ++i) pw[i] = st.plasticStrain[i];
            pw[6] = st.equivalentPlasticStrain;
            for (int i = 0; i < 6; ++i) m->stress[t * 6 + i] = sv[i];
            const double vol = m->rest_volume[t];
            dissipation += vol * inc.dissipation;
            const double pressure = (sv[0] + sv[1] + sv[2]) / 3.0;
            double density = 0;
            for (int i = 0; i < 3; ++i)
                density += 0.5 * sv[i] * ((sv[i] - pressure) / (2.0 * mu) + pressure / (3.0 * bulk));
            for (int i = 3; i < 6; ++i) density += 0.5 * sv[i] * (sv[i] / mu);
            strainEnergy += vol * density;

            M3d stress{};
            stress(0, 0) = sv[0];
            stress(1, 1) = sv[1];
            stress(2, 2) = sv[2];
            stress(0, 1) = stress(1, 0) = sv[3];
            stress(1, 2) = stress(2, 1) = sv[4];
            stress(2, 0) = stress(0, 2) = sv[5];
            const M3d piola = mul(r, stress);
            const M3d h = mul(piola, tr(dmInv));
            const double scale = -vol;
            double* out = &m->tet_force[t * 12];
            double f0[3] = {0, 0, 0};
            for (int c = 0; c < 3; ++c)
                for (int a = 0; a < 3; ++a) {
                    const double v = scale * h(a, c);
                    out[(c + 1) * 3 + a] = v;
                    f0[a] -= v;
                }
            for (int a = 0; a < 3; ++a) out[a] = f0[a];
        }
        double work = 0.0, gwork = 0.0, kinetic = 0.0;
        for (size_t n = 0; n < m->nodes; ++n) {
            if (m->fixed[n]) {
                for (int k = 0; k < 3; ++k) m->velocity[n * 3 + k] = 0.0;
                continue;
            }
            double force[3] = {0.0, 0.0, -p->gravity * m->mass[n]};
            for (uint32_t e = m->adj_offset[n]; e < m->adj_offset[n + 1]; ++e) {
                const uint32_t entry = m->adj_entry[e];
                const double* fs = &m->tet_force[(entry >> 2) * 12 + (entry & 3u) * 3];
                for (int k = 0; k < 3; ++k) force[k] += fs[k];
            }
            double ext[3] = {0.0, 0.0, 0.0};
            if (m->fext)
                for (int k = 0; k < 3; ++k) ext[k] = lf * m->fext[n * 3 + k];
            for (int k = 0; k < 3; ++k) force[k] += ext[k];
            const double invMass = 1.0 / m->mass[n];
            for (int k = 0; k < 3; ++k) {
                double v = m->velocity[n * 3 + k] + force[k] * invMass * p->dt;
                v *= p->damping;
                m->velocity[n * 3 + k] = v;
                m->position[n * 3 + k] += v * p->dt;
                work += ext[k] * v * p->dt;
                kinetic += 0.5 * m->mass[n] * v * v;
            }
            gwork += -p->gravity * m->mass[n] * m->velocity[n * 3 + 2] * p->dt;
        }
        m->energy[0] += work;
        m->energy[1] += dissipation;
        m->energy[2] = strainEnergy;
        m->energy[3] = kinetic;
        m->energy[4] += gwork;
        ++m->step;
    }
}

// One O-tet64 step of mesh m with the element loop spread over the workers of `jobs`
// by the reference's own core::JobSystem::parallelFor (as zone.cpp:967-973 spreads its
// element loop) and the node loop serial in CSR order (fem.cpp:196-214).  Per-tet
// energies go to `diss` and are summed in element order, so the result is the same for
// every worker count.
static void tet64_parallel_step(or_tet64* m, const or_tet64_params* p, const pl::Material& mat,
                                core::JobSystem& jobs, std::vector<double>& diss) {
    const double lf =
        p->ramp_steps > 0
            ? std::min(static_cast<double>(m->step + 1) / static_cast<double>(p->ramp_steps), 1.0)
            : 1.0;
    jobs.parallelFor(0, m->tets, 256, [&](std::size_t b, std::size_t e_end) {
        for (std::size_t t = b; t < e_end; ++t) {
            const uint32_t* idx = &m->index[t * 4];
            const double* x = m->position;
            M3d ds{};
            for (int c = 0; c < 3; ++c)
                for (int a = 0; a < 3; ++a) ds(a, c) = x[idx[c + 1] * 3 + a] - x[idx[0] * 3 + a];
            M3d dmInv{};
            for (int k = 0; k < 9; ++k) dmInv.m[k] = m->rest_inv[t * 9 + k];
            const M3d f = mul(ds, dmInv);
            const M3d r = polar(f, p->polar_fixed);
            const M3d sm = mul(tr(r), f);
            double strain[6];
            strain[0] = 0.5 * (sm(0, 0) + sm(0, 0)) - 1.0;
            strain[1] = 0.5 * (sm(1, 1) + sm(1, 1)) - 1.0;
            strain[2] = 0.5 * (sm(2, 2) + sm(2, 2)) - 1.0;
            strain[3] = 2.0 * (0.5 * (sm(0, 1) + sm(1, 0)));
            strain[4] = 2.0 * (0.5 * (sm(1, 2) + sm(2, 1)));
            strain[5] = 2.0 * (0.5 * (sm(2, 0) + sm(0, 2)));
            pl::State st;
            double* ps = &m->plastic[t * 7];
            for (int i = 0; i < 6; ++i) st.plasticStrain[i] = ps[i];
            st.equivalentPlasticStrain = ps[6];
            double sv[6];
            const pl::Increment inc = pl::update(mat, pl::kNeverFails, strain, st, sv);
            for (int i = 0; i < 6; ++i) ps[i] = st.plasticStrain[i];
            ps[6] = st.equivalentPlasticStrain;
            diss[t] = m->rest_volume[t] * inc.dissipation;
            M3d stress{};
            stress(0, 0) = sv[0];
            stress(1, 1) = sv[1];
            stress(2, 2) = sv[2];
            stress(0, 1) = stress(1, 0) = sv[3];
            stress(1, 2) = stress(2, 1) = sv[4];
            stress(2, 0) = stress(0, 2) = sv[5];
            const M3d h = mul(mul(r, stress), tr(dmInv));
            const double scale = -m->rest_volume[t];
            double* out = &m->tet_force[t * 12];
            double f0[3] = {0, 0, 0};
            for (int c = 0; c < 3; ++c)
                for (int a = 0; a < 3; ++a) {
                    const double v = scale * h(a, c);
                    out[(c + 1) * 3 + a] = v;
                    f0[a] -= v;
                }
            for (int a = 0; a < 3; ++a) out[a] = f0[a];
        }
    });
    for (size_t t = 0; t < m->tets; ++t) m->energy[1] += diss[t];
    for (size_t n = 0; n < m->nodes; ++n) {
        if (m->fixed[n]) {
            for (int k = 0; k < 3; ++k) m->velocity[n * 3 + k] = 0.0;
            continue;
        }
        double force[3] = {0.0, 0.0, -p->gravity * m->mass[n]};
        for (uint32_t e = m->adj_offset[n]; e < m->adj_offset[n + 1]; ++e) {
            const uint32_t entry = m->adj_entry[e];
            const double* fs = &m->tet_force[(entry >> 2) * 12 + (entry & 3u) * 3];
            for (int k = 0; k < 3; ++k) force[k] += fs[k];
        }
        if (m->fext)
            for (int k = 0; k < 3; ++k) force[k] += lf * m->fext[n * 3 + k];
        const double invMass = 1.0 / m->mass[n];
        for (int k = 0; k < 3; ++k) {
            double v = m->velocity[n * 3 + k] + force[k] * invMass * p->dt;
            v *= p->damping;
            m->velocity[n * 3 + k] = v;
            m->position[n * 3 + k] += v * p->dt;
        }
    }
    ++m->step;
}

static pl::Material tet64_material(const or_tet64_params* p) {
    pl::Material mat;
    mat.youngsModulus = p->E;
    mat.poissonRatio = p->nu;
    mat.flow = pl::linearHardening(p->yield, p->hardening);
    return mat;
}

// `steps` O-tet64 steps of one mesh over `workers` host threads.  Returns tets x steps
// / second of the step loop's own clock (thread start-up excluded).
double ref_tet64_time_parallel(or_tet64* m, const or_tet64_params* p, int steps, int workers) {
    const pl::Material mat = tet64_material(p);
    core::JobSystem jobs(workers > 1 ? static_cast<unsigned>(workers - 1) : 0u);
    std::vector<double> diss(m->tets);
    const auto begin = std::chrono::steady_clock::now();
    for (int s = 0; s < steps; ++s) tet64_parallel_step(m, p, mat, jobs, diss);
    const auto end = std::chrono::steady_clock::now();
    return static_cast<double>(m->tets) * steps / std::chrono::duration<double>(end - begin).count();
}

// `steps` steps of a batch of independent meshes, as the reference solves them: one
// mesh at a time (it steps one mesh per solver, fem.cpp:187), each mesh's element loop
// over `workers` host threads.  Step s of every mesh is taken before step s + 1 of any,
// so one timed step is one time step of the whole batch.  Returns the seconds of the
// step loop's own clock (thread start-up excluded).
double ref_tet64_time_batch(or_tet64* const* meshes, const or_tet64_params* params, size_t count, int steps,
                            int workers) {
    std::vector<pl::Material> mats;
    size_t most = 0;
    for (size_t i = 0; i < count; ++i) {
        mats.push_back(tet64_material(&params[i]));
        most = std::max(most, meshes[i]->tets);
    }
    core::JobSystem jobs(workers > 1 ? static_cast<unsigned>(workers - 1) : 0u);
    std::vector<double> diss(most);
    const auto begin = std::chrono::steady_clock::now();
    for (int s = 0; s < steps; ++s)
        for (size_t i = 0; i < count; ++i) tet64_parallel_step(meshes[i], &params[i], mats[i], jobs, diss);
    const auto end = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(end - begin).count();
}

// --- solid-shell -------------------------------------------------------------

int ref_shell_forms(const double rest[24], int formulation, double out[OR_FORMS_LEN]) {
    ss::RestForms f{};
    const bool ok = ss::computeRestForms(rest, formOf(formulation), f);
    formsOut(f, out);
    return ok ? 1 : 0;
}

void ref_shell_mass(const double nodes[24], double density, double out[8]) {
    ss::elementMass(nodes, density, out);
}

void ref_shell_gauss_volumes(const double nodes[24], double out[8]) {
    ss::gaussVolumes(nodes, out);
}

void ref_shell_init_state(const double nodes[24], const double* mat, double state[OR_SHELL_STATE_LEN]) {
    ss::ElementPlasticState st;
    ss::initialisePlasticState(nodes, toMaterial(mat), st);
    shellStateOut(st, state);
}

int ref_shell_plastic_update(const double forms[OR_FORMS_LEN], const double rest[24],
                             const double current[24], const double* mat,
                             double state[OR_SHELL_STATE_LEN], double force[24], double stress[48],
                             double info[7]) {
    ss::RestForms f{};
    formsIn(forms, f);
    ss::ElementPlasticState st;
    shellStateIn(state, st);
    const ss::PlasticUpdate u =
        ss::elementPlasticUpdate(f, rest, current, toMaterial(mat), st, force, stress);
    shellStateOut(st, state);
    if (info) {
        info[0] = u.converged;
        info[1] = u.iterations;
        info[2] = u.yieldedPoints;
        info[3] = u.failedPoints;
        info[4] = u.dissipation;
        info[5] = u.enhancedResidual;
        info[6] = u.enhancedWork;
    }
    return u.converged ? 1 : 0;
}

void ref_shell_rotation(const double forms[OR_FORMS_LEN], const double current[24], double out[9]) {
    ss::RestForms f{};
    formsIn(forms, f);
    ss::elementRotation(f, current, out);
}

void ref_shell_stiffness(const double nodes[24], double E, double nu, int formulation,
                         double out[576]) {
    sim::StructuralMaterial m;
    m.youngsModulus = E;
    m.poissonRatio = nu;
    ss::elementStiffness(nodes, m, formOf(formulation), out);
}

double ref_shell_critical_dt(const double nodes[24], double E, double nu, double rho,
                             int formulation, double safety) {
    sim::StructuralMaterial m;
    m.youngsModulus = E;
    m.poissonRatio = nu;
    m.density = rho;
    return ss::criticalTimestep(nodes, m, formOf(formulation), safety);
}

void ref_plate_sizes(int nx, int ny, int nz, size_t* nodes, size_t* elements) {
    *nodes = static_cast<size_t>(nx + 1) * (ny + 1) * (nz + 1);
    *elements = static_cast<size_t>(nx) * ny * nz;
}

void ref_plate_mesh(double lx, double ly, double thickness, int nx, int ny, int nz,
                    double* position, uint32_t* index) {
    const ss::HexMesh h = ss::makePlateMesh(lx, ly, thickness, nx, ny, nz);
    std::copy(h.position.begin(), h.position.end(), position);
    std::copy(h.index.begin(), h.index.end(), index);
}

void ref_plate_pressure_load(const double* position, const uint32_t* index, size_t nodes,
                             size_t elements, double pressure, double* load) {
    ss::HexMesh h;
    h.position.assign(position, position + nodes * 3);
    h.index.assign(index, index + elements * 8);
    const std::vector<double> l = ss::uniformPressureLoad(h, pressure);
    std::copy(l.begin(), l.end(), load);
}

// The zone set-up the solver constructor performs (zone.cpp:698-754): forms, mass,
// plastic state, Gauss volumes, CSR.
void ref_shell_setup(or_shell* m, const double* mat, double density) {
    const pl::Material material = toMaterial(mat);
    for (size_t n = 0; n < m->nodes; ++n) m->mass[n] = 0.0;
    for (size_t e = 0; e < m->elements; ++e) {
        double nodes[24];
        for (int a = 0; a < 8; ++a)
            for (int i = 0; i < 3; ++i) nodes[a * 3 + i] = m->rest[m->index[e * 8 + a] * 3 + i];
        ss::RestForms f{};
        ss::computeRestForms(nodes, ss::Formulation::SolidShell, f);
        formsOut(f, m->forms + e * OR_FORMS_LEN);
        double lumped[8];
        ss::elementMass(nodes, density, lumped);
        for (int a = 0; a < 8; ++a) m->mass[m->index[e * 8 + a]] += lumped[a];
        ss::ElementPlasticState st;
        ss::initialisePlasticState(nodes, material, st);
        shellStateOut(st, m->state + e * OR_SHELL_STATE_LEN);
        ss::gaussVolumes(nodes, m->gauss_volume + e * 8);
    }
    std::vector<uint32_t> off(m->nodes + 1, 0u);
    for (size_t e = 0; e < m->elements; ++e)
        for (int a = 0; a < 8; ++a) ++off[m->index[e * 8 + a] + 1];
    for (size_t i = 0; i < m->nodes; ++i) off[i + 1] += off[i];
    std::copy(off.begin(), off.end(), m->adj_offset);
    std::vector<uint32_t> cursor(off.begin(), off.end() - 1);
    for (size_t e = 0; e < m->elements; ++e)
        for (uint32_t a = 0; a < 8; ++a)
            m->adj_entry[cursor[m->index[e * 8 + a]]++] = static_cast<uint32_t>(e) * 8 + a;
}

// One explicit step as zone::Solver::step runs it for a patch with no punch and no
// driven edge (zone.cpp:928-989, 1094-1121, 1200-1202), with an external nodal load
// added to the gathered force.
void ref_shell_step(or_shell* m, const double* mat, const or_shell_params* p, int steps) {
    const pl::Material material = toMaterial(mat);
    for (int s = 0; s < steps; ++s) {
        const double time = static_cast<double>(m->step + 1) * p->dt;
        const double lf = p->rise_time > 0 ? std::min(time / p->rise_time, 1.0) : 1.0;
        double dissipation = 0.0;
        for (size_t e = 0; e < m->elements; ++e) {
            double rest[24], current[24];
            for (int a = 0; a < 8; ++a)
                for (int i = 0; i < 3; ++i) {
                    rest[a * 3 + i] = m->rest[m->index[e * 8 + a] * 3 + i];
                    current[a * 3 + i] = m->position[m->index[e * 8 + a] * 3 + i];
                }
            double* st = m->state + e * OR_SHELL_STATE_LEN;
            double* out = m->element_force + e * 24;
            double* stress = m->stress + e * 48;
            if (st[128] != 0.0) {
                std::fill(out, out + 24, 0.0);
                std::fill(stress, stress + 48, 0.0);
                continue;
            }
            ss::RestForms f{};
            formsIn(m->forms + e * OR_FORMS_LEN, f);
            ss::ElementPlasticState state;
            shellStateIn(st, state);
            const ss::PlasticUpdate u =
                ss::elementPlasticUpdate(f, rest, current, material, state, out, stress);
            shellStateOut(state, st);
            dissipation += u.dissipation;
        }
        double work = 0.0;
        for (size_t node = 0; node < m->nodes; ++node) {
            double sum[3] = {0, 0, 0};
            for (uint32_t k = m->adj_offset[node]; k < m->adj_offset[node + 1]; ++k) {
                const uint32_t entry = m->adj_entry[k];
                const double* f = &m->element_force[(entry / 8) * 24 + (entry % 8) * 3];
                sum[0] += f[0];
                sum[1] += f[1];
                sum[2] += f[2];
            }
            for (int k = 0; k < 3; ++k) {
                const size_t d = node * 3 + k;
                const double ext = m->fext ? lf * m->fext[d] : 0.0;
                const double force = sum[k] + ext;
                if (m->pinned[d]) {
                    m->velocity[d] = 0.0;
                    continue;
                }
                if (m->mass[node] > 0) m->velocity[d] += force / m->mass[node] * p->dt;
                m->velocity[d] *= p->damping;
                work += ext * m->velocity[d] * p->dt;
            }
        }
        for (size_t d = 0; d < m->nodes * 3; ++d) m->position[d] += m->velocity[d] * p->dt;
        m->energy[0] += work;
        m->energy[1] += dissipation;
        ++m->step;
    }
}

// --- zone::Solver itself --------------------------------------------------------

namespace {

void materialOut(const pl::Material& m, double* out) {
    out[0] = m.youngsModulus;
    out[1] = m.poissonRatio;
    out[2] = m.flow.yieldStrength;
    out[3] = m.flow.hardeningModulus;
    out[4] = m.flow.kinematicModulus;
    out[5] = m.flow.kind == pl::Hardening::Swift ? 1.0 : 0.0;
    out[6] = m.flow.strengthCoefficient;
    out[7] = m.flow.referenceStrain;
    out[8] = m.flow.hardeningExponent;
    out[9] = m.failure.uniformStrain;
    out[10] = m.failure.fractureStrain;
    out[11] = m.failure.triaxialitySensitivity;
    out[12] = m.failure.referenceTriaxiality;
    out[13] = m.failure.cutoffTriaxiality;
}

// The plate patch of the reference's zone GPU tests (tests/test_zone_gpu.cpp:163-197),
// with a driven perimeter when edge_drive is non-zero.
sim::zone::Patch platePatch(const or_zone_case* c) {
    ss::HexMesh flat = ss::makePlateMesh(c->lx, c->ly, c->thickness, c->nx, c->ny, c->nz);
    flat.prescribed.assign(flat.nodeCount() * 3, 0.0);
    for (std::size_t n = 0; n < flat.nodeCount(); ++n) {
        const double x = flat.position[n * 3], y = flat.position[n * 3 + 1];
        if (x <= 1e-9 || x >= c->lx - 1e-9 || y <= 1e-9 || y >= c->ly - 1e-9)
            for (int k = 0; k < 3; ++k) flat.pin(n, k, c->edge_drive[k] * (x / c->lx));
    }
    sim::zone::Patch patch;
    patch.mesh = flat;
    patch.axis = sim::Vec3{0, 0, 1};
    patch.right = sim::Vec3{1, 0, 0};
    patch.up = sim::Vec3{0, 1, 0};
    patch.centre = sim::Vec3{0.5 * c->lx, 0.5 * c->ly, 0.0};
    patch.outerFace.assign(flat.nodeCount(), 0u);
    for (std::size_t n = 0; n < flat.nodeCount(); ++n)
        patch.outerFace[n] = flat.position[n * 3 + 2] > 0.0 ? 1u : 0u;
    patch.elementArea.assign(flat.elementCount(), c->lx * c->ly / (double)(c->nx * c->ny));
    patch.panelOf.assign(flat.elementCount(), 0);
    patch.panels.push_back(0);
    patch.panelArea.push_back(c->lx * c->ly);
    patch.material = sim::ah36Steel();
    patch.thickness = c->thickness;
    patch.criticalTimestep =
        ss::criticalTimestep(flat, patch.material, ss::Formulation::SolidShell);
    // flat-bar stiffeners along x on grid lines, the web on the -z side
    if (c->stiffeners > 0) {
        patch.stiffening.material = sim::ah36Steel();
        const int nzp = c->nz + 1;
        for (int s = 0; s < c->stiffeners; ++s) {
            const int j = (int)std::lround((double)c->ny * (s + 1) / (c->stiffeners + 1));
            sim::constraint::SeamRun run;
            run.sign = -1.0;
            for (int i = 0; i <= c->nx; ++i) {
                const uint32_t base = (uint32_t)((i * (c->ny + 1) + j) * nzp);
                run.bottom.push_back(base);
                run.top.push_back(base + (uint32_t)c->nz);
            }
            sim::constraint::addStiffener(run, sim::flatBar(c->web_height, c->web_thickness), c->thickness,
                                          patch.mesh.position, patch.stiffening);
        }
    }
    return patch;
}

sim::zone::SolveParams plateParams(const or_zone_case* c) {
    sim::zone::SolveParams params;
    params.indenter.halfLength = c->half_length;
    params.indenter.halfWidth = c->half_width;
    params.indenter.speed = c->speed;
    params.indenter.rampTime = c->mass > 0 ? 0.0 : c->ramp_time;
    params.indenter.stopAt = 1.0;
    if (c->mass > 0) {
        params.indenter.drive = sim::zone::Drive::Inertial;
        params.indenter.mass = c->mass;
    }
    params.damping = c->damping;
    params.edgeRamp = c->edge_ramp;
    params.fiberFailure = c->fiber_failure != 0;
    return params;
}

}  // namespace

extern "C" int ref_zone_sizes(const or_zone_case* c, size_t out[3]) {
    const sim::zone::Patch patch = platePatch(c);
    out[0] = patch.nodeCount();
    out[1] = patch.elementCount();
    out[2] = patch.stiffening.fiberCount();
    return 0;
}

// Build the plate, construct zone::Solver on it and call step() `steps` times; return
// the arrays the solver was built from and where it ended.  Returns the number of
// problems the solver reported.
extern "C" int ref_zone_run(const or_zone_case* c, or_zone_out* o) {
    const sim::zone::Patch patch = platePatch(c);
    const sim::zone::SolveParams params = plateParams(c);
    const pl::Material material = pl::shipSteel();
    sim::zone::Solver solver(patch, material, params);
    const std::size_t N = patch.nodeCount(), E = patch.elementCount();
    std::copy(patch.mesh.position.begin(), patch.mesh.position.end(), o->rest);
    std::copy(patch.mesh.index.begin(), patch.mesh.index.end(), o->index);
    std::copy(solver.pinnedDof().begin(), solver.pinnedDof().end(), o->pinned);
    std::copy(patch.mesh.prescribed.begin(), patch.mesh.prescribed.end(), o->prescribed);
    std::fill(o->driven, o->driven + N, uint8_t{0});
    for (uint32_t n : solver.drivenNodes()) o->driven[n] = 1;
    std::copy(solver.nodalMass().begin(), solver.nodalMass().end(), o->mass);
    for (std::size_t e = 0; e < E; ++e) shellStateOut(solver.elementState()[e], o->state0 + e * OR_SHELL_STATE_LEN);
    materialOut(material, o->mat);
    o->density = patch.material.density;
    for (int s = 0; s < c->steps; ++s)
        if (!solver.step()) break;
    const sim::zone::SolveResult& r = solver.result();
    o->dt = r.timestep;
    std::copy(solver.position().begin(), solver.position().end(), o->position);
    std::copy(solver.velocity().begin(), solver.velocity().end(), o->velocity);
    for (std::size_t e = 0; e < E; ++e) shellStateOut(solver.elementState()[e], o->state + e * OR_SHELL_STATE_LEN);
    const double account[10] = {r.work, r.dissipation, r.penetration, r.time, r.dampingLoss, r.boundaryWork,
                                r.indenterSpeed, (double)r.steps, r.indenterArrested ? 1.0 : 0.0,
                                (double)r.drivenEdgeDof};
    std::copy(account, account + 10, o->account);
    // the fibres as the solver holds them (zone.cpp:724-733): rest lengths from rest_,
    // each fibre's own failure strain, and their state after the steps
    const sim::constraint::Stiffening& st = patch.stiffening;
    const sim::constraint::RestFibers forms = sim::constraint::restFibers(st, solver.rest());
    for (std::size_t i = 0; i < st.fiberCount(); ++i) {
        const sim::constraint::Fiber& f = st.fiber[i];
        o->fiber_tie[i * 4] = f.end[0].bottom;
        o->fiber_tie[i * 4 + 1] = f.end[0].top;
        o->fiber_tie[i * 4 + 2] = f.end[1].bottom;
        o->fiber_tie[i * 4 + 3] = f.end[1].top;
        o->fiber_weight[i * 2] = f.end[0].weight;
        o->fiber_weight[i * 2 + 1] = f.end[1].weight;
        o->fiber_area[i] = f.area;
        o->fiber_length[i] = forms.length[i];
        o->fiber_fail[i] = params.fiberFailure
                               ? sim::constraint::fiberFailureStrain(material.failure, forms.length[i], f.neckWidth)
                               : pl::kNeverFails;
        const sim::constraint::FiberState zero{};
        const sim::constraint::FiberState& fs = i < solver.fiberState().size() ? solver.fiberState()[i] : zero;
        o->fiber_state[i * 4] = fs.plasticStrain;
        o->fiber_state[i * 4 + 1] = fs.equivalentPlasticStrain;
        o->fiber_state[i * 4 + 2] = fs.damage;
        o->fiber_state[i * 4 + 3] = fs.failed ? 1.0 : 0.0;
    }
    return (int)r.problems.size();
}

// zone.cpp:1014-1044 (kinetic and the plastic strain energy).
void ref_shell_energy(or_shell* m, const double* mat) {
    const pl::Material material = toMaterial(mat);
    const double mu = material.shearModulus(), bulk = material.bulkModulus();
    double kinetic = 0;
    for (size_t node = 0; node < m->nodes; ++node) {
        const double* v = &m->velocity[node * 3];
        kinetic += 0.5 * m->mass[node] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    }
    double strain = 0;
    for (size_t e = 0; e < m->elements; ++e)
        for (int gp = 0; gp < 8; ++gp) {
            const double* s = &m->stress[e * 48 + gp * 6];
            const double pressure = (s[0] + s[1] + s[2]) / 3.0;
            double density = 0;
            for (int i = 0; i < 3; ++i)
                density += 0.5 * s[i] * ((s[i] - pressure) / (2.0 * mu) + pressure / (3.0 * bulk));
            for (int i = 3; i < 6; ++i) density += 0.5 * s[i] * (s[i] / mu);
            strain += m->gauss_volume[e * 8 + gp] * density;
        }
    m->energy[2] = strain;
    m->energy[3] = kinetic;
}

// zone::Solver::step's element loop over all host cores with core::JobSystem
// (zone.cpp:967-973), for the CPU baseline timing.  Returns elements x steps / s.
double ref_shell_time_parallel(or_shell* m, const double* mat, const or_shell_params* p,
                               int steps, int workers) {
    const pl::Material material = toMaterial(mat);
    core::JobSystem jobs(workers > 0 ? static_cast<unsigned>(workers)
                                     : core::JobSystem::defaultWorkerCount());
    std::vector<ss::RestForms> forms(m->elements);
    for (size_t e = 0; e < m->elements; ++e) formsIn(m->forms + e * OR_FORMS_LEN, forms[e]);
    std::vector<ss::ElementPlasticState> plastic(m->elements);
    for (size_t e = 0; e < m->elements; ++e) shellStateIn(m->state + e * OR_SHELL_STATE_LEN, plastic[e]);
    const auto begin = std::chrono::steady_clock::now();
    for (int s = 0; s < steps; ++s) {
        const double time = static_cast<double>(m->step + 1) * p->dt;
        const double lf = p->rise_time > 0 ? std::min(time / p->rise_time, 1.0) : 1.0;
        jobs.parallelFor(0, m->elements, 8, [&](std::size_t b, std::size_t e_end) {
            for (std::size_t e = b; e < e_end; ++e) {
                double rest[24], current[24];
                for (int a = 0; a < 8; ++a)
                    for (int i = 0; i < 3; ++i) {
                        rest[a * 3 + i] = m->rest[m->index[e * 8 + a] * 3 + i];
                        current[a * 3 + i] = m->position[m->index[e * 8 + a] * 3 + i];
                    }
                ss::elementPlasticUpdate(forms[e], rest, current, material, plastic[e],
                                         m->element_force + e * 24, m->stress + e * 48);
            }
        });
        for (size_t node = 0; node < m->nodes; ++node) {
            double sum[3] = {0, 0, 0};
            for (uint32_t k = m->adj_offset[node]; k < m->adj_offset[node + 1]; ++k) {
                const uint32_t entry = m->adj_entry[k];
                const double* f = &m->element_force[(entry / 8) * 24 + (entry % 8) * 3];
                sum[0] += f[0];
                sum[1] += f[1];
                sum[2] += f[2];
            }
            for (int k = 0; k < 3; ++k) {
                const size_t d = node * 3 + k;
                const double ext = m->fext ? lf * m->fext[d] : 0.0;
                if (m->pinned[d]) {
                    m->velocity[d] = 0.0;
                    continue;
                }
                if (m->mass[node] > 0) m->velocity[d] += (sum[k] + ext) / m->mass[node] * p->dt;
            }
        }
        for (size_t d = 0; d < m->nodes * 3; ++d) m->position[d] += m->velocity[d] * p->dt;
        ++m->step;
    }
    const auto end = std::chrono::steady_clock::now();
    const double seconds = std::chrono::duration<double>(end - begin).count();
    return static_cast<double>(m->elements) * steps / seconds;
}

unsigned ref_default_workers(void) { return core::JobSystem::defaultWorkerCount() + 1; }

// fem::stepCpu timed alone (single-threaded by design): tets x steps / second.
double ref_tet32_time(or_tet32* m, float E, float nu, float rho, float dt, int steps) {
    fem::TetMesh t = toTetMesh(m);
    fem::Material mat;
    mat.youngsModulus = E;
    mat.poissonRatio = nu;
    mat.density = rho;
    const auto begin = std::chrono::steady_clock::now();
    for (int s = 0; s < steps; ++s) fem::stepCpu(t, mat, dt, 0.0f, 1.0f);
    const auto end = std::chrono::steady_clock::now();
    fromTetMesh(t, m);
    return static_cast<double>(m->tets) * steps / std::chrono::duration<double>(end - begin).count();
}

}  // extern "C"
