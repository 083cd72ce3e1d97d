// pool.cu -- kernels of the multi-mesh pool (pool.hpp): the batched and served step.
//
// Every block works on one tile: a run of one mesh's tets (or nodes).  The mesh's
// parameters come from its record; a mesh whose step count is reached is frozen
// (its tiles do nothing) until the host retires it.  The energy partial of a tile goes
// to the slot its mesh was given at admission, so nothing in a mesh's result depends
// on what else is in the pool.
#include <algorithm>

#include "bulk.cuh"
#include "common.cuh"
#include "omega.cuh"
#include "pool.hpp"
#include "tet.hpp"

namespace fs {
namespace {

__device__ __forceinline__ TetElementRefs element_refs(const PoolDevice& d) {
    return TetElementRefs{d.index,     d.slot, d.rest_inv, d.rest_vol, d.plastic,
                          d.plastic_c, d.disp, d.disp_c,   d.slots,    d.tet_cap};
}

__device__ __forceinline__ TetNodeRefs node_refs(const PoolDevice& d) {
    return TetNodeRefs{d.offset, d.slots, d.fixed, d.mass, d.inv_mass, d.ext, d.velocity, d.disp, d.disp_c};
}

// One element tile at sub-step `sub` of the chunk (all threads of the block call it).
// CG: data other blocks wrote earlier in the same launch is read through L2.
// `ahead`: the tile this block prefetches into L2 (the one a wave later), or -1.
template <bool CG>
__device__ __forceinline__ void element_tile(const PoolDevice& d, int tile, int sub, double* scratch, int ahead) {
    if (ahead >= 0 && ahead < d.n_etiles) {
        const PoolTile nx = d.etiles[ahead];
        prefetch_tet_rows(element_refs(d), nx.begin, nx.end);
    }
    const PoolTile tl = d.etiles[tile];
    const PoolMesh& m = d.meshes[tl.mesh];
    const bool live = m.step + sub < m.target;
    double diss = 0.0, energy = 0.0;
    const long long t = tl.begin + threadIdx.x;
    if (live && t < tl.end) tet_element_f32<true, CG>(element_refs(d), t, m.mat, diss, energy);
    block_sum2(diss, energy, scratch);  // valid in thread 0
    if (live && threadIdx.x == 0) {
        d.e_diss[tl.part] += diss;
        d.e_strain[tl.part] = energy;
    }
}

template <bool CG>
__device__ __forceinline__ void node_tile(const PoolDevice& d, int tile, int sub, double* scratch) {
    const PoolTile tl = d.ntiles[tile];
    const PoolMesh& m = d.meshes[tl.mesh];
    const long long step = m.step + sub;
    const bool live = step < m.target;
    double work = 0.0, kin = 0.0, gwork = 0.0;
    const long long n = tl.begin + threadIdx.x;
    if (live && n < tl.end) {
        const float lf = (float)ramp_factor(step, m.ramp);
        tet_node_f32<true, CG>(node_refs(d), n, lf, m.dt, m.gravity, m.damping, work, kin, gwork);
    }
    work += gwork;
    block_sum2(work, kin, scratch);  // valid in thread 0
    if (live && threadIdx.x == 0) {
        d.n_work[tl.part] += work;
        d.n_kin[tl.part] = kin;
    }
}

// B threads per block (the tile); 1024 / B blocks per SM bound the element pass to 64
// registers, 32 resident warps per SM whatever the tile.
// `wave`: the blocks resident on the whole GPU at once; block b prefetches tile b + wave.
template <int B>
__global__ void __launch_bounds__(B, 1024 / B) pool_elements(PoolDevice d, int sub, int wave) {
    __shared__ double scratch[64];
    element_tile<false>(d, blockIdx.x, sub, scratch, blockIdx.x + wave);
}

// The bound on a wait for a tile's staged rows: a few million polls (seconds), far
// beyond any copy's time; a wait that runs out is reported, never waited out.
constexpr uint32_t kStageWaitPolls = 1u << 22;

// The element pass on a persistent grid with each tile's own rows staged into shared
// memory one tile ahead: block b takes tiles b, b + grid, b + 2 grid, ...  While the
// block computes one tile, its thread 0 has already queued the bulk copies of the next
// tile's rows (node ids, slot map, Dm^-1, volume, plastic state: the 19 copies of
// stage_tile_rows) into the other of two buffers, completed on that buffer's mbarrier.
// So the rows' DRAM latency runs behind a whole tile's arithmetic, and a tet finds its
// own rows in shared memory; only the corner displacements are read from global
// memory (mostly L1 hits: the tets of a tile share their nodes).  A buffer is refilled
// only after the barrier that ends the tile which read it.  Waits are bounded: a tile
// whose copies do not land sets the pool's error flag and is skipped, and the launch
// still ends (the host then reports FEMSTEP_ETIMEOUT and retires the pool).  The
// arithmetic is tet_element_f32's, so the results are the plain pass's to the bit.
template <int B>
struct RingStage {
    static constexpr int kPitch = B + 4;
    uint4 idx[B];
    uint4 slot[B];
    float rows[17 * kPitch];
};

// Thread 0: queue the copies of `tile`'s rows into stage `st` (or arrive with nothing,
// for a frozen mesh's tile).
template <int B>
__device__ __forceinline__ void stage_tile_rows(const PoolDevice& d, int tile, int sub, RingStage<B>& st,
                                                uint64_t* bar) {
    const PoolTile tl = d.etiles[tile];
    const PoolMesh& m = d.meshes[tl.mesh];
    if (!(m.step + sub < m.target)) {
        mbar_arrive(bar);
        return;
    }
    const long long first = tl.begin, n = tl.end - tl.begin;
    const long long base = first & ~3LL, last4 = (tl.end + 3) & ~3LL;
    const uint32_t row_bytes = (uint32_t)((last4 - base) * 4);
    mbar_arrive_expect_tx(bar, 2u * (uint32_t)n * 16u + 17u * row_bytes);
    bulk_copy_g2s(st.idx, d.index + first, (uint32_t)n * 16u, bar);
    bulk_copy_g2s(st.slot, d.slot + first, (uint32_t)n * 16u, bar);
    for (int k = 0; k < 9; ++k)
        bulk_copy_g2s(st.rows + k * RingStage<B>::kPitch, d.rest_inv + (size_t)k * d.tet_cap + base, row_bytes, bar);
    bulk_copy_g2s(st.rows + 9 * RingStage<B>::kPitch, d.rest_vol + base, row_bytes, bar);
    for (int i = 0; i < 7; ++i)
        bulk_copy_g2s(st.rows + (10 + i) * RingStage<B>::kPitch, d.plastic + (size_t)i * d.tet_cap + base, row_bytes,
                      bar);
}

// MINB: the blocks per SM the register budget is set for.
template <int B, int MINB>
__global__ void __launch_bounds__(B, MINB) pool_elements_ring(PoolDevice d, int sub) {
    __shared__ double scratch[64];
    __shared__ __align__(8) uint64_t bar[2];
    extern __shared__ __align__(16) unsigned char ring_smem[];  // two RingStage<B>
    RingStage<B>* stage = reinterpret_cast<RingStage<B>*>(ring_smem);
    const TetElementRefs r = element_refs(d);
    const int stride = (int)gridDim.x;
    int tile = blockIdx.x;
    if (tile >= d.n_etiles) return;  // the whole block (the grid is at most the tile count)
    uint32_t issued[2] = {0u, 0u};   // thread 0: the phases it queued on each buffer
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        stage_tile_rows<B>(d, tile, sub, stage[0], &bar[0]);
        issued[0] = 1;
    }
    __syncthreads();  // the barriers are set up before anyone waits on them
    for (int k = 0;; ++k) {
        const int b = k & 1;
        const int next = tile + stride;
        // once a wait anywhere has given up, nothing more is staged or waited for
        const bool failed = *(volatile int*)d.error != 0;
        // the other buffer was last read by the tile before this one, which the
        // previous iteration's closing barrier has finished
        if (threadIdx.x == 0 && next < d.n_etiles && !failed) {
            stage_tile_rows<B>(d, next, sub, stage[b ^ 1], &bar[b ^ 1]);
            ++issued[b ^ 1];
        }
        const PoolTile tl = d.etiles[tile];
        const PoolMesh& m = d.meshes[tl.mesh];
        const bool live = m.step + sub < m.target;
        // buffer b's (k / 2)-th phase holds this tile
        const bool ok = !failed && mbar_wait_bounded(&bar[b], (uint32_t)((k >> 1) & 1), kStageWaitPolls);
        if (!ok && !failed) atomicExch(d.error, 1);
        double diss = 0.0, energy = 0.0;
        const long long t = tl.begin + threadIdx.x;
        if (ok && live && t < tl.end) {
            const long long base = tl.begin & ~3LL;
            tet_element_f32<true, false, SharedRows>(
                r, SharedRows{stage[b].idx, stage[b].slot, stage[b].rows, RingStage<B>::kPitch, tl.begin, base}, t,
                m.mat, diss, energy);
        }
        block_sum2(diss, energy, scratch);  // valid in thread 0; also the closing barrier
        if (threadIdx.x == 0 && live && ok) {
            d.e_diss[tl.part] += diss;
            d.e_strain[tl.part] = energy;
        }
        if (next >= d.n_etiles) break;
        tile = next;
    }
    // after a wait gave up, copies may still be in flight into this block's shared
    // memory: thread 0 lets the last phase of each buffer land (bounded) before the
    // block, and with it its shared memory, retires
    if (threadIdx.x == 0 && *(volatile int*)d.error != 0) {
        for (int b = 0; b < 2; ++b)
            if (issued[b]) mbar_wait_bounded(&bar[b], (issued[b] - 1) & 1, kStageWaitPolls);
    }
}

// Up to 2048 / B blocks per SM (32 registers): the pass waits on its loads, and twice
// the warps of the element pass hide more of that (0.093 -> 0.079 ms on the 256-mesh
// batch in the tiled schedule).
template <int B>
__global__ void __launch_bounds__(B, 2048 / B) pool_nodes(PoolDevice d, int sub) {
    __shared__ double scratch[64];
    node_tile<false>(d, blockIdx.x, sub, scratch);
}

// Every active mesh advances by the steps it took in the chunk.
__global__ void pool_advance(PoolDevice d, int steps) {
    for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < d.n_active; i += blockDim.x * gridDim.x) {
        PoolMesh* m = d.meshes + d.active[i];
        if (m->step < m->target) {
            const long long next = m->step + steps;
            m->step = next < m->target ? next : m->target;
        }
    }
}

// Grid-wide barrier for the persistent launch, bounded: a block that waits longer
// than ~0.5 s sets the error flag and goes on, and every later barrier then gives up
// at once, so the launch always ends.  The launch is cooperative, so all blocks are
// co-resident and the wait is never expected to run out.
__device__ __forceinline__ bool grid_sync(unsigned int* bar, unsigned int nblocks, int* err) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int* gen = bar + 1;
        const unsigned int g = *gen;
        __threadfence();
        if (atomicAdd(bar, 1u) == nblocks - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            unsigned long long spins = 0;
            while (*gen == g) {
                if (*(volatile int*)err != 0 || ++spins > (1ull << 24)) {
                    atomicExch(err, 1);
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *(volatile int*)err == 0;
}

template <int B>
__global__ void __launch_bounds__(B, 1024 / B) pool_persistent(PoolDevice d, int steps) {
    __shared__ double scratch[64];
    for (int s = 0; s < steps; ++s) {
        for (int tile = blockIdx.x; tile < d.n_etiles; tile += gridDim.x)
            element_tile<true>(d, tile, s, scratch, tile + (int)gridDim.x);
        if (!grid_sync(d.barrier, gridDim.x, d.error)) return;
        for (int tile = blockIdx.x; tile < d.n_ntiles; tile += gridDim.x) node_tile<true>(d, tile, s, scratch);
        if (!grid_sync(d.barrier, gridDim.x, d.error)) return;
    }
}


}  // namespace

// The staged pass's two stages in dynamic shared memory (52 KB for tiles of 256, above
// the 48 KB a launch gets without asking), and its persistent grid: as many blocks as
// fit on the GPU at once, at most one per tile.
template <int B>
static size_t ring_smem_bytes() {
    return 2 * sizeof(RingStage<B>);
}

// Eight blocks of 128 per SM (four of 256): 64 registers per thread and 32 warps.  A
// budget of six blocks (80 registers, no spill) measured 7 % slower: the warps hide
// more latency than the spilled registers cost.
template <int B>
constexpr int kRingBlocks = 1024 / B;

template <int B>
static int ring_grid(int tiles) {
    static int per_sm = -1;
    if (per_sm < 0) {
        cudaFuncSetAttribute(pool_elements_ring<B, kRingBlocks<B>>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)ring_smem_bytes<B>());
        int n = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, pool_elements_ring<B, kRingBlocks<B>>, B,
                                                      ring_smem_bytes<B>());
        per_sm = n > 0 ? n : 1;
    }
    return std::min(tiles, per_sm * sm_count());
}

void pool_kernels_setup() {
    ring_grid<128>(1);
    ring_grid<256>(1);
}

void launch_pool_element_pass(const PoolDevice& d, int tile, int sub, cudaStream_t stream, bool staged) {
    if (!d.n_etiles) return;
    if (staged && tile == 128) {
        pool_elements_ring<128, kRingBlocks<128>>
            <<<ring_grid<128>(d.n_etiles), 128, ring_smem_bytes<128>(), stream>>>(d, sub);
        return;
    }
    if (staged && tile == 256) {
        pool_elements_ring<256, kRingBlocks<256>>
            <<<ring_grid<256>(d.n_etiles), 256, ring_smem_bytes<256>(), stream>>>(d, sub);
        return;
    }
    const int wave = sm_count() * (1024 / tile);
    switch (tile) {
        case 128: pool_elements<128><<<d.n_etiles, 128, 0, stream>>>(d, sub, wave); break;
        case 256: pool_elements<256><<<d.n_etiles, 256, 0, stream>>>(d, sub, wave); break;
        default: pool_elements<512><<<d.n_etiles, 512, 0, stream>>>(d, sub, wave); break;
    }
}

void launch_pool_node_pass(const PoolDevice& d, int tile, int sub, cudaStream_t stream) {
    if (!d.n_ntiles) return;
    switch (tile) {
        case 128: pool_nodes<128><<<d.n_ntiles, 128, 0, stream>>>(d, sub); break;
        case 256: pool_nodes<256><<<d.n_ntiles, 256, 0, stream>>>(d, sub); break;
        default: pool_nodes<512><<<d.n_ntiles, 512, 0, stream>>>(d, sub); break;
    }
}

void launch_pool_steps(const PoolDevice& d, int tile, int steps, cudaStream_t stream, PoolPasses passes) {
    if (d.n_etiles == 0 || steps <= 0) return;
    // the tiled node pass gathers the per-tile partials through their own CSR
    PoolDevice dn = d;
    if (passes == PoolPasses::kTiled) dn.offset = const_cast<uint32_t*>(d.part_off);
    for (int s = 0; s < steps; ++s) {
        if (passes == PoolPasses::kTiled)
            launch_pool_tiled_element_pass(d, s, stream);
        else
            launch_pool_element_pass(d, tile, s, stream, passes == PoolPasses::kStaged);
        launch_pool_node_pass(dn, tile, s, stream);
    }
    pool_advance<<<blocks_for(d.n_active, 256), 256, 0, stream>>>(d, steps);
}

void launch_pool_advance(const PoolDevice& d, int steps, cudaStream_t stream) {
    if (d.n_active) pool_advance<<<blocks_for(d.n_active, 256), 256, 0, stream>>>(d, steps);
}

int pool_persistent_max_blocks(int tile) {
    int per_sm = 0, sms = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    switch (tile) {
        case 128: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pool_persistent<128>, 128, 0); break;
        case 256: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pool_persistent<256>, 256, 0); break;
        default: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pool_persistent<512>, 512, 0); break;
    }
    return per_sm * sms;
}

cudaError_t launch_pool_persistent(const PoolDevice& d, int tile, int steps, int blocks, cudaStream_t stream) {
    if (d.n_etiles == 0 || steps <= 0) return cudaSuccess;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(tile);
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e;
    switch (tile) {
        case 128: e = cudaLaunchKernelEx(&cfg, pool_persistent<128>, d, steps); break;
        case 256: e = cudaLaunchKernelEx(&cfg, pool_persistent<256>, d, steps); break;
        default: e = cudaLaunchKernelEx(&cfg, pool_persistent<512>, d, steps); break;
    }
    if (e != cudaSuccess) return e;
    pool_advance<<<blocks_for(d.n_active, 256), 256, 0, stream>>>(d, steps);
    return cudaGetLastError();
}

namespace {

// The rest state of an admitted mesh on the device, in FP64 as the single-mesh handle
// computes it on the host (fem.cpp:119-158): per tet Dm^-1 and the volume, stored as
// float rows, and the tet's quarter of its lumped mass parked in the first 8 bytes of
// each corner's force slot (the element pass writes every slot before anything reads
// it).  The mesh's rest positions are staged in its own velocity rows (indexed by
// pool node id), which the admission zeroes afterwards.
__device__ __forceinline__ void rest_tet(const PoolDevice& d, long long t0, long long t, double density) {
    const float* pos = d.velocity;
    const uint4 id4 = d.index[t0 + t];
    const uint32_t id[4] = {id4.x, id4.y, id4.z, id4.w};
    double a[9];  // column-major, as the host
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r)
            a[c * 3 + r] = (double)pos[(size_t)id[c + 1] * 3 + r] - (double)pos[(size_t)id[0] * 3 + r];
#define A(r, c) a[(c) * 3 + (r)]
    const double det = A(0, 0) * (A(1, 1) * A(2, 2) - A(1, 2) * A(2, 1)) -
                       A(0, 1) * (A(1, 0) * A(2, 2) - A(1, 2) * A(2, 0)) +
                       A(0, 2) * (A(1, 0) * A(2, 1) - A(1, 1) * A(2, 0));
    const double volume = fabs(det / 6.0);
    const double inv_det = fabs(det) > 1e-300 ? 1.0 / det : 0.0;
    double r[9];
#define R(rr, cc) r[(cc) * 3 + (rr)]
    R(0, 0) = (A(1, 1) * A(2, 2) - A(1, 2) * A(2, 1)) * inv_det;
    R(0, 1) = (A(0, 2) * A(2, 1) - A(0, 1) * A(2, 2)) * inv_det;
    R(0, 2) = (A(0, 1) * A(1, 2) - A(0, 2) * A(1, 1)) * inv_det;
    R(1, 0) = (A(1, 2) * A(2, 0) - A(1, 0) * A(2, 2)) * inv_det;
    R(1, 1) = (A(0, 0) * A(2, 2) - A(0, 2) * A(2, 0)) * inv_det;
    R(1, 2) = (A(0, 2) * A(1, 0) - A(0, 0) * A(1, 2)) * inv_det;
    R(2, 0) = (A(1, 0) * A(2, 1) - A(1, 1) * A(2, 0)) * inv_det;
    R(2, 1) = (A(0, 1) * A(2, 0) - A(0, 0) * A(2, 1)) * inv_det;
    R(2, 2) = (A(0, 0) * A(1, 1) - A(0, 1) * A(1, 0)) * inv_det;
#undef R
#undef A
    for (int k = 0; k < 9; ++k) d.rest_inv[(size_t)k * d.tet_cap + t0 + t] = (float)r[k];
    d.rest_vol[t0 + t] = (float)volume;
    const double quarter = density * volume * 0.25;
    const uint4 sl = d.slot[t0 + t];
    const uint32_t slot[4] = {sl.x, sl.y, sl.z, sl.w};
    for (int c = 0; c < 4; ++c) *reinterpret_cast<double*>(d.slots + slot[c]) = quarter;
}

// Lumped node masses: the tets' quarters over the node's CSR run, which lists its tets
// in ascending order -- the order the host loop adds them in.  Then the spare node.
__device__ __forceinline__ void rest_node(const PoolDevice& d, long long n0, long long N, long long n) {
    if (n == N) {  // the spare node slot holds the CSR end and has no mass
        d.mass[n0 + N] = 0.0f;
        d.inv_mass[n0 + N] = 0.0f;
        return;
    }
    double m = 0.0;
    for (uint32_t k = d.offset[n0 + n]; k < d.offset[n0 + n + 1]; ++k) m += *reinterpret_cast<const double*>(d.slots + k);
    d.mass[n0 + n] = (float)m;
    d.inv_mass[n0 + n] = m > 0.0 ? (float)(1.0 / m) : 0.0f;
}

// The group record a thread's item belongs to: the last one whose prefix `first` of the
// kind given is <= k (records ascend).
template <long long PoolAdmit::*First>
__device__ __forceinline__ int admit_of(const PoolAdmit* adm, int G, long long k) {
    int lo = 0, hi = G - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (adm[mid].*First <= k)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Per tet of the group: zero its plastic state, form its rest state.  Per partial
// slot of the group: zero the four energy partials.
__global__ void pool_admit_tets(PoolDevice d, const PoolAdmit* adm, int G, long long tets, long long parts) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < tets; k += stride) {
        const PoolAdmit& a = adm[admit_of<&PoolAdmit::tet_first>(adm, G, k)];
        const long long t = k - a.tet_first;
        for (int i = 0; i < 7; ++i) {
            d.plastic[(size_t)i * d.tet_cap + a.t0 + t] = 0.0f;
            d.plastic_c[(size_t)i * d.tet_cap + a.t0 + t] = 0.0f;
        }
        rest_tet(d, a.t0, t, a.density);
    }
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < parts; k += stride) {
        const PoolAdmit& a = adm[admit_of<&PoolAdmit::part_first>(adm, G, k)];
        const long long q = a.part0 + (k - a.part_first);
        d.e_diss[q] = 0.0;
        d.e_strain[q] = 0.0;
        d.n_work[q] = 0.0;
        d.n_kin[q] = 0.0;
    }
}

// Per node of the group (and each mesh's spare slot): its lumped mass from the tets'
// quarters, then displacement, compensation and velocity at rest (the velocity rows
// held the staged positions until now).
__global__ void pool_admit_nodes(PoolDevice d, const PoolAdmit* adm, int G, long long nodes) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nodes; k += stride) {
        const PoolAdmit& a = adm[admit_of<&PoolAdmit::node_first>(adm, G, k)];
        const long long n = k - a.node_first;
        rest_node(d, a.n0, a.N, n);
        d.disp[a.n0 + n] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        d.disp_c[a.n0 + n] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        float* v = d.velocity + (size_t)(a.n0 + n) * 3;
        v[0] = v[1] = v[2] = 0.0f;
    }
}

// Per tet of a mesh that wants its step formed: the element bound from the stored
// FP32 Dm^-1 (promoted to double), maximised per mesh.  A non-negative double orders
// as its bit pattern, so the maximum is an integer atomicMax and exact.
__global__ void pool_admit_omega(PoolDevice d, const PoolAdmit* adm, int G, long long tets,
                                 unsigned long long* w2) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < tets; k += stride) {
        const int g = admit_of<&PoolAdmit::tet_first>(adm, G, k);
        const PoolAdmit& a = adm[g];
        if (!a.want_dt) continue;
        const long long t = a.t0 + (k - a.tet_first);
        double gr[4][3];
        for (int c = 0; c < 3; ++c)
            for (int r = 0; r < 3; ++r) gr[c + 1][r] = (double)d.rest_inv[(size_t)(r * 3 + c) * d.tet_cap + t];
        for (int r = 0; r < 3; ++r) gr[0][r] = -(gr[1][r] + gr[2][r] + gr[3][r]);
        const double v = tet_omega2_one<true>(gr, a.lambda, a.mu, a.density);
        atomicMax(w2 + g, (unsigned long long)__double_as_longlong(v > 0.0 ? v : 0.0));
    }
}

__global__ void pool_admit_dt(PoolMesh* meshes, const PoolAdmit* adm, int G, const unsigned long long* w2) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G || !adm[g].want_dt) return;
    const double v = __longlong_as_double((long long)w2[g]);
    const double dt = v > 0.0 ? 0.9 * 2.0 / sqrt(v) : 0.0;  // safety 0.9, as the single-mesh bound
    meshes[adm[g].id].dt64 = dt;
    meshes[adm[g].id].dt = (float)dt;
}

}  // namespace

namespace {
__global__ void pool_rebase(uint4* index, long long tets, uint32_t add) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tets; t += (long long)gridDim.x * blockDim.x) {
        uint4 v = index[t];
        v.x += add;
        v.y += add;
        v.z += add;
        v.w += add;
        index[t] = v;
    }
}
}  // namespace

void launch_pool_rebase(uint4* index, long long tets, uint32_t add, cudaStream_t stream) {
    if (tets > 0) pool_rebase<<<std::min<long long>(blocks_for(tets, 256), 148 * 16), 256, 0, stream>>>(index, tets, add);
}

void launch_pool_admit(const PoolDevice& d, const PoolAdmit* adm, int G, long long tets, long long nodes,
                       long long parts, bool any_dt, unsigned long long* w2, cudaStream_t stream) {
    const int cap = sm_count() * 8;
    auto grid = [&](long long n) { return (int)std::max(1LL, std::min((long long)cap, (n + kBlock - 1) / kBlock)); };
    pool_admit_tets<<<grid(std::max(tets, parts)), kBlock, 0, stream>>>(d, adm, G, tets, parts);
    pool_admit_nodes<<<grid(nodes), kBlock, 0, stream>>>(d, adm, G, nodes);
    if (any_dt) {
        cudaMemsetAsync(w2, 0, (size_t)G * sizeof(unsigned long long), stream);
        pool_admit_omega<<<grid(tets), kBlock, 0, stream>>>(d, adm, G, tets, w2);
        pool_admit_dt<<<(G + 127) / 128, 128, 0, stream>>>(d.meshes, adm, G, w2);
    }
}



}  // namespace fs
