// compat/zone_gpu.cpp -- gpu::ZoneGpuSolver over libfemstep.so (see engine/gpu/zone_gpu.hpp
// in this directory).
#include "engine/gpu/zone_gpu.hpp"

#include <cmath>
#include <cstdint>
#include <vector>

#include "engine/sim/constraint.hpp"
#include "femstep.h"

namespace gpu {

namespace {

// ElementPlasticState <-> the 129 doubles of femstep_shell_state (zone_gpu.cpp:36-40).
void pack(const sim::solidshell::ElementPlasticState& s, double* x) {
    for (int gp = 0; gp < sim::solidshell::kGauss; ++gp) {
        const sim::plasticity::State& p = s.point[gp];
        double* y = x + gp * 15;
        for (int i = 0; i < 6; ++i) {
            y[i] = p.plasticStrain[i];
            y[6 + i] = p.backStress[i];
        }
        y[12] = p.equivalentPlasticStrain;
        y[13] = p.damage;
        y[14] = p.failed ? 1.0 : 0.0;
    }
    for (int k = 0; k < sim::solidshell::kEas; ++k) x[120 + k] = s.enhanced[k];
    x[127] = s.failureStrain;
    x[128] = s.torn ? 1.0 : 0.0;
}

void unpack(const double* x, sim::solidshell::ElementPlasticState& s) {
    for (int gp = 0; gp < sim::solidshell::kGauss; ++gp) {
        sim::plasticity::State& p = s.point[gp];
        const double* y = x + gp * 15;
        for (int i = 0; i < 6; ++i) {
            p.plasticStrain[i] = y[i];
            p.backStress[i] = y[6 + i];
        }
        p.equivalentPlasticStrain = y[12];
        p.damage = y[13];
        p.failed = y[14] != 0.0;
    }
    for (int k = 0; k < sim::solidshell::kEas; ++k) s.enhanced[k] = x[120 + k];
    s.failureStrain = x[127];
    s.torn = x[128] != 0.0;
}

}  // namespace

struct ZoneGpuSolver::Impl {
    femstep_shell* handle = nullptr;
    femstep_shell_params params{};
    femstep_shell_material material{};
    std::size_t nodes = 0, elements = 0;
};

std::string describeElementPipelines(const std::string& /*shaderDirectory*/) {
    return "libfemstep.so shell_forces: one element per 8 lanes of a warp (lane = Gauss point), FP32 with "
           "Kahan-compensated displacement and plastic strain, FP64 energy partials; the same kernel for both "
           "mappings (ptxas reports its registers and spills at build time)\n";
}

ZoneGpuSolver::~ZoneGpuSolver() {
    if (impl_) femstep_shell_destroy(impl_->handle);
    delete impl_;
}

bool ZoneGpuSolver::initialise(const sim::zone::Patch& patch, const sim::zone::Solver& cpu,
                               const sim::plasticity::Material& material, const sim::zone::SolveParams& params,
                               const std::string& /*shaderDirectory*/, std::string& error, Mapping mapping,
                               EasPrecision eas) {
    // the reference's own refusals (zone_gpu.cpp:500-517)
    if (cpu.restForms().size() != patch.elementCount()) {
        error = "the CPU solver was built without SolveParams::cacheRestForms, so there is nothing to upload";
        return false;
    }
    if (!params.plastic) {
        error = "the GPU path implements the elastoplastic element only";
        return false;
    }
    if (eas != EasPrecision::Float && mapping != Mapping::Workgroup) {
        error = "the fp64 enhanced-strain variants are compiled for the workgroup mapping only; the one-invocation "
                "kernel is float throughout";
        return false;
    }
    if (impl_) femstep_shell_destroy(impl_->handle);
    delete impl_;
    impl_ = new Impl();
    device_ = nullptr;
    Impl& d = *impl_;
    const std::size_t N = patch.nodeCount(), E = patch.elementCount();
    d.nodes = N;
    d.elements = E;

    // rest forms in zone_gpu.cpp's order: B [8][6][24], G [8][6][7], w [8], J0^-1 [9]
    std::vector<double> forms(E * 1505);
    for (std::size_t e = 0; e < E; ++e) {
        const sim::solidshell::RestForms& f = cpu.restForms()[e];
        double* x = forms.data() + e * 1505;
        for (int gp = 0; gp < 8; ++gp)
            for (int i = 0; i < 6; ++i) {
                for (int c = 0; c < 24; ++c) x[(gp * 6 + i) * 24 + c] = f.b[gp][i][c];
                for (int k = 0; k < 7; ++k) x[1152 + (gp * 6 + i) * 7 + k] = f.g[gp][i][k];
            }
        for (int gp = 0; gp < 8; ++gp) x[1488 + gp] = f.weight[gp];
        for (int k = 0; k < 9; ++k) x[1496 + k] = f.restJacobianInverse[k];
    }
    std::vector<double> state(E * 129);
    for (std::size_t e = 0; e < E; ++e) pack(cpu.elementState()[e], state.data() + e * 129);
    const std::vector<uint32_t> index(patch.mesh.index.begin(), patch.mesh.index.end());

    femstep_shell_mesh m{};
    m.nodes = N;
    m.elements = E;
    m.rest = cpu.rest().data();
    m.position = cpu.position().data();
    m.velocity = cpu.velocity().data();
    m.index = index.data();
    m.pinned = cpu.pinnedDof().data();
    m.load = nullptr;
    m.forms = forms.data();
    m.mass = cpu.nodalMass().data();
    m.state = state.data();
    m.adjacency_offset = cpu.adjacencyOffset().data();
    m.adjacency_entry = cpu.adjacencyEntry().data();
    m.density = 0.0;
    if (femstep_shell_create(&m, &d.handle) != FEMSTEP_OK) {
        error = femstep_last_error();
        d.handle = nullptr;
        return false;
    }

    // the point law
    const sim::plasticity::FlowCurve& flow = material.flow;
    d.material.hardening = flow.kind == sim::plasticity::Hardening::Swift ? FEMSTEP_SHELL_SWIFT : FEMSTEP_SHELL_LINEAR;
    d.material.strength_coefficient = flow.strengthCoefficient;
    d.material.reference_strain = flow.referenceStrain;
    d.material.hardening_exponent = flow.hardeningExponent;
    d.material.kinematic_modulus = flow.kinematicModulus;
    d.material.triaxiality_sensitivity = material.failure.triaxialitySensitivity;
    d.material.reference_triaxiality = material.failure.referenceTriaxiality;
    d.material.cutoff_triaxiality = material.failure.cutoffTriaxiality;
    femstep_shell_params& p = d.params;
    p.youngs_modulus = material.youngsModulus;
    p.poisson_ratio = material.poissonRatio;
    p.yield_strength = flow.yieldStrength;
    p.hardening_modulus = flow.hardeningModulus;
    // SolveParams::timestep, or the patch's critical step at timestepSafety (zone_gpu.cpp:526-527)
    p.dt = params.timestep > 0 ? params.timestep : patch.criticalTimestep * (params.timestepSafety / 0.9);
    p.damping = params.damping;
    p.rise_time = 0.0;
    // The ladder of zone_gpu.hpp:153-162, with the reference kernels' stopping rules
    // (solidshell_forces_wg.comp: ||r|| <= 1e-12 sigma_y V throughout; |delta . r| <=
    // 1e-9 sigma_y V in at most 12 iterations as shipped, the CPU's 1e-16 and 40 for the
    // tight float control and the fp64 Newton rung).  The FP64 rungs add double to the
    // 7x7 solve, then to the condensation, then to alpha itself.
    const bool tight = eas == EasPrecision::FloatTight || eas == EasPrecision::Newton;
    p.max_iterations = tight ? 40 : 12;
    p.tol_residual = 1e-12;
    p.tol_work = tight ? 1e-16 : 1e-9;
    p.compensated = 1;
    p.material = &d.material;
    p.eas_fp64 = eas == EasPrecision::Solve ? 1 : eas == EasPrecision::Condense ? 2 : eas == EasPrecision::Newton ? 3 : 0;

    // the punch: the CPU solver's driven nodes, along -axis; prescribed, or the striking
    // body of Drive::Inertial (zone.cpp:1154-1185)
    const std::vector<uint32_t> driven(cpu.drivenNodes().begin(), cpu.drivenNodes().end());
    const double axis[3] = {patch.axis.x, patch.axis.y, patch.axis.z};
    const double striker =
        params.indenter.drive == sim::zone::Drive::Inertial ? params.indenter.mass : 0.0;
    if (femstep_shell_set_punch(d.handle, driven.data(), driven.size(), axis, params.indenter.speed,
                                params.indenter.rampTime, striker) != FEMSTEP_OK) {
        error = femstep_shell_error(d.handle);
        return false;
    }
    // the driven edge: pinned DOFs with a prescribed value, measured from the meshed
    // position (zone.cpp:833-842, 1123-1145)
    if (patch.mesh.prescribed.size() == N * 3 &&
        femstep_shell_set_edge(d.handle, patch.mesh.prescribed.data(), patch.mesh.position.data(),
                               params.edgeRamp) != FEMSTEP_OK) {
        error = femstep_shell_error(d.handle);
        return false;
    }
    // the stiffeners as constraint fibres (zone.cpp:724-733, 990-1002): the rest
    // lengths from the CPU solver's rest array and each fibre's own failure strain; the
    // CPU solver's lumped mass already holds their mass
    const sim::constraint::Stiffening& st = patch.stiffening;
    if (!st.empty()) {
        const sim::constraint::RestFibers rest = sim::constraint::restFibers(st, cpu.rest());
        const std::size_t F = st.fiberCount();
        std::vector<uint32_t> tie(F * 4);
        std::vector<double> weight(F * 2), area(F), fail(F);
        for (std::size_t i = 0; i < F; ++i) {
            const sim::constraint::Fiber& f = st.fiber[i];
            tie[i * 4] = f.end[0].bottom;
            tie[i * 4 + 1] = f.end[0].top;
            tie[i * 4 + 2] = f.end[1].bottom;
            tie[i * 4 + 3] = f.end[1].top;
            weight[i * 2] = f.end[0].weight;
            weight[i * 2 + 1] = f.end[1].weight;
            area[i] = f.area;
            fail[i] = params.fiberFailure
                          ? sim::constraint::fiberFailureStrain(material.failure, rest.length[i], f.neckWidth)
                          : sim::plasticity::kNeverFails;
        }
        femstep_shell_fibers fibers{F, tie.data(), weight.data(), area.data(), rest.length.data(), fail.data(), 0.0};
        if (femstep_shell_set_fibers(d.handle, &fibers) != FEMSTEP_OK) {
            error = femstep_shell_error(d.handle);
            return false;
        }
    }
    char name[256] = {0};
    if (femstep_device_name(name, sizeof(name)) == FEMSTEP_OK) deviceName_ = name;
    static const char* const rung[5] = {
        "shell_forces (libfemstep.so, 8 lanes per element, FP32 compensated)",
        "shell_forces (libfemstep.so, 8 lanes per element, FP32 compensated, the CPU's stopping rule)",
        "shell_forces<EAS64=1> (libfemstep.so, 8 lanes per element, the 7x7 enhanced solve in FP64)",
        "shell_forces<EAS64=2> (libfemstep.so, 8 lanes per element, the enhanced condensation in FP64)",
        "shell_forces<EAS64=3> (libfemstep.so, 8 lanes per element, alpha and its Newton in FP64)"};
    elementShader_ = rung[static_cast<int>(eas)];
    device_ = d.handle;
    steps_ = 0;
    return true;
}

double ZoneGpuSolver::run(int substeps) {
    if (!impl_ || !impl_->handle) return -1.0;
    double ms = 0.0;
    if (femstep_shell_run(impl_->handle, substeps, &impl_->params, &ms) != FEMSTEP_OK) return -1.0;
    steps_ += substeps;
    return ms;
}

ZoneGpuState ZoneGpuSolver::readback() const {
    ZoneGpuState out;
    if (!impl_ || !impl_->handle) return out;
    const Impl& d = *impl_;
    out.position.resize(d.nodes * 3);
    out.velocity.resize(d.nodes * 3);
    femstep_shell_readback(d.handle, out.position.data(), out.velocity.data());
    std::vector<double> state(d.elements * 129);
    femstep_shell_state(d.handle, state.data());
    out.plastic.resize(d.elements);
    for (std::size_t e = 0; e < d.elements; ++e) {
        unpack(state.data() + e * 129, out.plastic[e]);
        if (out.plastic[e].torn) ++out.tornElements;
    }
    double energy[4] = {0, 0, 0, 0}, punch[4] = {0, 0, 0, 0};
    femstep_shell_energy(d.handle, energy);
    femstep_shell_punch_state(d.handle, punch);
    out.dissipation = energy[1];
    out.work = punch[0];
    out.penetration = punch[1];
    out.time = punch[2];
    out.steps = static_cast<int>(punch[3]);
    return out;
}

}  // namespace gpu
