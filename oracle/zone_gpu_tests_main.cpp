// Runs the reference's own GPU zone suite (tests/test_zone_gpu.cpp and its harness,
// compiled unchanged from the reference's tree by `make zone_gpu_tests`) against the
// drop-in gpu::ZoneGpuSolver of sinking-simulator_b200/compat over libfemstep.so.
// The reference's tests/main.cpp runs every suite of the project; this main runs the
// one suite for the GPU zone step and prints the harness's counts.
#include "harness.hpp"

#include <cstdio>

int main() {
    runZoneGpuTests();
    std::printf("\nzone_gpu suite: %d checks, %d failed\n", testing::checkCount(), testing::failureCount());
    return testing::failureCount() == 0 ? 0 : 1;
}
