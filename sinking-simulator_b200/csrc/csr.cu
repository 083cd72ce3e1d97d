// csr.cu -- the node -> corner adjacency (CSR) and the corner -> slot map, built on
// the device.
//
// The reference builds the adjacency on the CPU with a counting sort in element order
// (zone::Solver's adjacencyOffset / adjacencyEntry, engine/sim/zone.cpp:739-755): node
// n's run lists the corners e * 8 + c that name it, ascending.  Here: count the corners
// per node (atomic increments), an exclusive scan for the offsets, a scatter with
// atomic cursors, and then each node's run sorted ascending -- which makes the result
// independent of the scatter's order and identical to the CPU counting sort.  Runs are
// short (eight for an interior node of a hex mesh), so each node sorts its own run by
// insertion.  The slot map inverts the entries: slot[corner] = its position in the CSR.
// An entry naming a node id >= `nodes` is left out (no run, no slot): the pool's tiled
// tables pad their lists with such entries.
#include <cub/device/device_scan.cuh>

#include "common.cuh"
#include "shell.hpp"

namespace fs {
namespace {

__global__ void csr_count(const uint32_t* index, long long total, long long nodes, uint32_t* count) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x)
        if (index[i] < nodes) atomicAdd(&count[index[i]], 1u);
}

__global__ void csr_scatter(const uint32_t* index, long long total, long long nodes, uint32_t* cursor,
                            uint32_t* entry) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x)
        if (index[i] < nodes) entry[atomicAdd(&cursor[index[i]], 1u)] = (uint32_t)i;
}

__global__ void csr_sort_runs(const uint32_t* offset, long long nodes, uint32_t* entry) {
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nodes) return;
    const uint32_t b = offset[n], e = offset[n + 1];
    for (uint32_t k = b + 1; k < e; ++k) {
        const uint32_t v = entry[k];
        uint32_t j = k;
        while (j > b && entry[j - 1] > v) {
            entry[j] = entry[j - 1];
            --j;
        }
        entry[j] = v;
    }
}

// over the entries counted: offset[nodes] of them (before the base is added)
__global__ void csr_slots(const uint32_t* entry, const uint32_t* counted, uint32_t* slot, uint32_t base) {
    const long long total = *counted;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x)
        slot[entry[k]] = base + (uint32_t)k;
}

__global__ void csr_add_base(uint32_t* offset, long long n, uint32_t base) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        offset[i] += base;
}

}  // namespace

cudaError_t build_csr_device(const uint32_t* index, long long total, long long nodes, uint32_t* offset, uint32_t* slot,
                             cudaStream_t stream, uint32_t* entry_out, uint32_t base) {
    uint32_t *count = nullptr, *entry = entry_out;
    void* temp = nullptr;
    size_t temp_bytes = 0;
    cudaError_t err = cub::DeviceScan::InclusiveSum(nullptr, temp_bytes, count, offset + 1, (int)nodes, stream);
    if (err == cudaSuccess) err = cudaMallocAsync(&count, (size_t)nodes * sizeof(uint32_t), stream);
    if (err == cudaSuccess && !entry) err = cudaMallocAsync(&entry, (size_t)total * sizeof(uint32_t), stream);
    if (err == cudaSuccess) err = cudaMallocAsync(&temp, temp_bytes, stream);
    if (err == cudaSuccess) {
        const int grid = 148 * 8;
        cudaMemsetAsync(count, 0, (size_t)nodes * sizeof(uint32_t), stream);
        cudaMemsetAsync(offset, 0, sizeof(uint32_t), stream);
        csr_count<<<grid, 256, 0, stream>>>(index, total, nodes, count);
        err = cub::DeviceScan::InclusiveSum(temp, temp_bytes, count, offset + 1, (int)nodes, stream);
    }
    if (err == cudaSuccess) {
        // the cursors start at each run's first position: offset[0 .. nodes)
        cudaMemcpyAsync(count, offset, (size_t)nodes * sizeof(uint32_t), cudaMemcpyDeviceToDevice, stream);
        const int grid = 148 * 8;
        csr_scatter<<<grid, 256, 0, stream>>>(index, total, nodes, count, entry);
        csr_sort_runs<<<blocks_for(nodes, 256), 256, 0, stream>>>(offset, nodes, entry);
        csr_slots<<<grid, 256, 0, stream>>>(entry, offset + nodes, slot, base);
        if (base) csr_add_base<<<grid, 256, 0, stream>>>(offset, nodes + 1, base);
        err = cudaGetLastError();
    }
    if (temp) cudaFreeAsync(temp, stream);
    if (entry && entry != entry_out) cudaFreeAsync(entry, stream);
    if (count) cudaFreeAsync(count, stream);
    return err;
}

}  // namespace fs
