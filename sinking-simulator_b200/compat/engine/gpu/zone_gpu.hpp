// engine/gpu/zone_gpu.hpp -- drop-in replacement of the reference's Vulkan zone back-end.
//
// Same types and public interface as solarbaron/sinking-simulator's
// engine/gpu/zone_gpu.hpp (ZoneGpuState, Mapping, EasPrecision,
// describeElementPipelines, ZoneGpuSolver), implemented over libfemstep.so's C ABI
// (femstep_shell_*).  Put this directory ahead of the engine sources on the include
// path and link compat/zone_gpu.cpp and libfemstep.so in place of
// engine/gpu/zone_gpu.cpp; callers such as tools/zone_gpu_probe compile unchanged.
//
// Behaviour kept from the reference (zone_gpu.cpp:495-985):
//   - initialise takes everything from the CPU solver it is handed (rest, position,
//     velocity, lumped mass, pinned DOF, rest forms, element state with each element's
//     failure strain, the CSR, the driven nodes) and returns false with a reason
//     instead of throwing -- on no device, on a solver built without cached rest
//     forms, on an elastic-only solve, and on a combination it does not build;
//   - the step is the element update (the general point law: linear or Swift flow,
//     kinematic hardening, ductile damage, the degraded-EAS retry, tearing), the CSR
//     gather, the node update with its damping, the driven edge and the punch, all on
//     the device.  Beyond the reference's GPU path, which drives a prescribed punch
//     only: the inertial punch (Drive::Inertial) and the driven edge run here too;
//   - run executes `substeps` steps with the host out of the loop and returns the
//     device-measured milliseconds; readback returns the ZoneGpuState that
//     zone::Solver::adopt takes.
// What differs: the element runs in FP32 with Kahan-compensated displacement and
// plastic strain and an FP64 energy account; both mappings run the same 8-lanes-per-
// element kernel; the fp64 enhanced-strain variants (Solve / Condense / Newton) are not
// built and initialise says so; `shaderDirectory` is accepted and ignored.
#pragma once

#include "engine/sim/plasticity.hpp"
#include "engine/sim/zone.hpp"

#include <string>
#include <vector>

struct femstep_shell;

namespace gpu {

struct ZoneGpuState {
    std::vector<double> position;
    std::vector<double> velocity;
    std::vector<sim::solidshell::ElementPlasticState> plastic;
    double work = 0;         // J the punch put in, accumulated on the device
    double dissipation = 0;  // J plastic, accumulated on the device
    int steps = 0;
    double time = 0;
    double penetration = 0;
    int tornElements = 0;
};

enum class Mapping {
    Invocation,
    Workgroup,
};

enum class EasPrecision {
    Float,
    FloatTight,
    Solve,
    Condense,
    Newton,
};

std::string describeElementPipelines(const std::string& shaderDirectory);

class ZoneGpuSolver {
public:
    ~ZoneGpuSolver();
    ZoneGpuSolver() = default;
    ZoneGpuSolver(const ZoneGpuSolver&) = delete;
    ZoneGpuSolver& operator=(const ZoneGpuSolver&) = delete;

    bool initialise(const sim::zone::Patch& patch, const sim::zone::Solver& cpu,
                    const sim::plasticity::Material& material, const sim::zone::SolveParams& params,
                    const std::string& shaderDirectory, std::string& error, Mapping mapping = Mapping::Workgroup,
                    EasPrecision eas = EasPrecision::Float);

    double run(int substeps);

    ZoneGpuState readback() const;

    const std::string& deviceName() const { return deviceName_; }
    const std::string& elementShader() const { return elementShader_; }
    bool valid() const { return device_ != nullptr; }
    int steps() const { return steps_; }

private:
    struct Impl;
    Impl* impl_ = nullptr;
    void* device_ = nullptr;  // the femstep_shell handle, for valid()
    std::string deviceName_;
    std::string elementShader_;
    int steps_ = 0;
};

}  // namespace gpu
