// compat/fem_gpu.cpp -- gpu::FemGpuSolver over libfemstep.so (see engine/gpu/fem_gpu.hpp
// in this directory).
#include "engine/gpu/fem_gpu.hpp"

#include "femstep.h"

namespace gpu {

FemGpuSolver::~FemGpuSolver() { femstep_tet_destroy(handle_); }

bool FemGpuSolver::initialise(const sim::fem::TetMesh& mesh, const std::string& /*shaderDirectory*/,
                              std::string& error) {
    femstep_tet_destroy(handle_);
    handle_ = nullptr;
    femstep_tet_mesh m{};
    m.nodes = mesh.nodeCount();
    m.tets = mesh.tetCount();
    m.position = mesh.position.data();
    m.velocity = mesh.velocity.empty() ? nullptr : mesh.velocity.data();
    m.mass = mesh.mass.data();
    m.fixed = mesh.fixed.empty() ? nullptr : mesh.fixed.data();
    m.index = mesh.index.data();
    m.rest_inv = mesh.restInv.data();
    m.rest_volume = mesh.restVolume.data();
    m.adjacency_offset = mesh.adjacencyOffset.data();
    m.adjacency_entry = mesh.adjacencyEntry.data();
    const int rc = femstep_tet_create(&m, FEMSTEP_TET_REF32, &handle_);
    if (rc != FEMSTEP_OK) {
        error = femstep_last_error();
        handle_ = nullptr;
        return false;
    }
    char name[256] = {0};
    if (femstep_device_name(name, sizeof(name)) == FEMSTEP_OK) deviceName_ = name;
    return true;
}

double FemGpuSolver::run(int substeps, const sim::fem::Material& material, float dt, float gravity, float damping) {
    femstep_tet_params p{};
    p.youngs_modulus = material.youngsModulus;
    p.poisson_ratio = material.poissonRatio;
    p.dt = dt;
    p.gravity = gravity;
    p.damping = damping;
    double ms = 0.0;
    if (femstep_tet_run(handle_, substeps, &p, &ms) != FEMSTEP_OK) return -1.0;
    return ms;
}

void FemGpuSolver::readback(sim::fem::TetMesh& mesh) {
    femstep_tet_readback(handle_, mesh.position.data(), mesh.velocity.data());
}

}  // namespace gpu
