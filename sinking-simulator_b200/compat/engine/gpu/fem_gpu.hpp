// engine/gpu/fem_gpu.hpp -- drop-in replacement of the reference's Vulkan tet back-end.
//
// Same class, same public interface as solarbaron/sinking-simulator's
// engine/gpu/fem_gpu.hpp:17-45, implemented over libfemstep.so's C ABI
// (include/femstep.h, FEMSTEP_TET_REF32).  Put this directory ahead of the engine
// sources on the include path and link compat/fem_gpu.cpp and libfemstep.so in place
// of engine/gpu/fem_gpu.cpp; callers such as tools/fem_spike compile unchanged.
//
// Behaviour kept from the reference:
//   - initialise returns false with a reason on any failure, including "no device",
//     so callers skip rather than fail (fem_gpu.hpp:21-22);
//   - run executes `substeps` steps with the host out of the loop and returns the
//     device-measured milliseconds (fem_gpu.hpp:26-32);
//   - readback copies positions and velocities into the caller's mesh (:34-35).
// What differs: the arithmetic is fem::stepCpu's to the bit (the Vulkan shaders only
// agreed to 1e-4 after one step, tools/fem_spike/main.cpp:207-210), and the
// `shaderDirectory` argument is accepted and ignored -- the kernels are in the library.
#pragma once

#include "engine/sim/fem.hpp"

#include <string>

struct femstep_tet;

namespace gpu {

class FemGpuSolver {
public:
    FemGpuSolver() = default;
    ~FemGpuSolver();
    FemGpuSolver(const FemGpuSolver&) = delete;
    FemGpuSolver& operator=(const FemGpuSolver&) = delete;

    bool initialise(const sim::fem::TetMesh& mesh, const std::string& shaderDirectory, std::string& error);
    double run(int substeps, const sim::fem::Material& material, float dt, float gravity, float damping);
    void readback(sim::fem::TetMesh& mesh);

    const std::string& deviceName() const { return deviceName_; }
    bool valid() const { return handle_ != nullptr; }

private:
    femstep_tet* handle_ = nullptr;
    std::string deviceName_;
};

}  // namespace gpu
