// pool.hpp -- a resident pool of many independent J2 tet meshes, stepped together.
//
// The batched and the served workloads (many meshes of uneven size, each with its own
// material, load, time step and step count) share one device pool:
//
//   * tets and nodes of every admitted mesh live in contiguous ranges of pool-wide
//     structure-of-arrays (the same per-tet / per-node layout as the single mesh,
//     tet.hpp), allocated first-fit against the pool's capacity;
//   * the work is a list of tiles, each a run of up to `tile` tets (or nodes) of ONE
//     mesh, so a block never mixes meshes and each mesh's arithmetic -- including
//     the fixed-order energy partial of each of its own tiles -- is the same whatever
//     else is in the pool;
//   * a chunk of `steps` steps is an element pass and a node pass per step, then one
//     advance of every mesh's step counter by the steps it took.  During a chunk the
//     counters are read only: sub-step s of a mesh at step k is step k + s, live while
//     k + s < target.  The passes run either as two launches per step (replayed from
//     a captured CUDA graph) or inside one persistent launch with two bounded grid
//     barriers per step.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "tet_f32.cuh"

namespace fs {

struct PoolMesh {           // device-side per-mesh record
    J2f mat;
    float dt, gravity, damping;
    int ramp;               // load ramp in steps
    long long step;         // steps taken
    long long target;       // steps requested; the mesh is frozen once step == target
    long long e_part, n_part;  // first energy-partial slot of its element / node tiles
    double dt64;            // the time step before rounding to float
    long long serial;       // admission number: tells a record from an earlier tenant's
};

struct PoolTile {           // a run of one mesh's tets or nodes
    int mesh;
    int part;               // energy-partial slot
    long long begin, end;   // pool indices
};

struct PoolDevice {
    long long tet_cap = 0, node_cap = 0;
    // tets (SoA, stride tet_cap)
    uint4* index = nullptr;
    uint4* slot = nullptr;
    float* rest_inv = nullptr;
    float* rest_vol = nullptr;
    float* plastic = nullptr;
    float* plastic_c = nullptr;
    float4* slots = nullptr;       // 4 per tet capacity: (fx, fy, fz, 0) per corner
    // nodes
    uint32_t* offset = nullptr;    // [node_cap]: CSR begin of each node; every mesh holds
                                   // one spare node slot after its last node for the end
    float4* disp = nullptr;        // (ux, uy, uz, 0)
    float4* disp_c = nullptr;
    float* velocity = nullptr;
    float* mass = nullptr;
    float* inv_mass = nullptr;
    uint8_t* fixed = nullptr;
    float* ext = nullptr;
    // meshes and work
    PoolMesh* meshes = nullptr;
    const PoolTile* etiles = nullptr;
    const PoolTile* ntiles = nullptr;
    int n_etiles = 0, n_ntiles = 0;
    const int* active = nullptr;   // ids of the meshes in the work lists
    int n_active = 0;
    // FP64 energy partials, per tile slot (fixed per mesh for its lifetime):
    // dissipation (+=), strain energy (=), external work incl. gravity (+=), kinetic (=)
    double* e_diss = nullptr;
    double* e_strain = nullptr;
    double* n_work = nullptr;
    double* n_kin = nullptr;
    // The tiled schedule's tables (built for the work list at tile 128; null otherwise).
    // Per element tile g: its distinct nodes, ascending, at node_tab[tab_off[g] ..
    // tab_off[g] + tab_count[g]) (each tile's list padded to a multiple of 8 entries, so
    // it starts on a 16-byte boundary); per tet its corners' places in that list (lidx,
    // four 16-bit ids); the tile's corners sorted by node and then by tet (inv, at 4 x
    // the tet's pool index, each given as its place c x 128 + i in the element pass's
    // force buffer, corner c of tet i of the tile); per listed node the start of its
    // corners in inv (inv_start) and the slot of its per-tile force partial (part_slot).
    // part_off: the node-major CSR over those partials, ascending tile within each
    // node's run; the partials go in `slots`.
    const uint32_t* tab_off = nullptr;
    const uint32_t* tab_count = nullptr;
    const uint32_t* node_tab = nullptr;
    const uint16_t* inv_start = nullptr;
    const uint32_t* part_slot = nullptr;
    const ushort4* lidx = nullptr;
    const uint16_t* inv = nullptr;
    const uint32_t* part_off = nullptr;
    int tab_kcap = 0;  // the staged tiled pass's stage size: the largest tile's node count, to a multiple of 8
    unsigned int* barrier = nullptr;  // [0] arrivals, [1] generation
    int* error = nullptr;             // set by a grid barrier that gave up waiting
};

// How a step's element pass runs: direct; with each tile's rows staged in shared
// memory by bulk async copies (tiles of 128 and 256; a 512 tile runs the direct pass);
// or tiled (tiles of 128: per-tile node gather and per-(tile, node) force partials).
enum class PoolPasses { kDirect, kStaged, kTiled };
// Two launches per step (element, node), `steps` times, then the advance, on `stream`.
void launch_pool_steps(const PoolDevice& d, int tile, int steps, cudaStream_t stream, PoolPasses passes);
// The passes one at a time (per-kernel timing): element or node pass of sub-step
// `sub`, and the advance by `steps`.
void launch_pool_element_pass(const PoolDevice& d, int tile, int sub, cudaStream_t stream, bool staged);
void launch_pool_node_pass(const PoolDevice& d, int tile, int sub, cudaStream_t stream);
void launch_pool_advance(const PoolDevice& d, int steps, cudaStream_t stream);
// One persistent cooperative launch for `steps` steps on `blocks` co-resident blocks,
// then the advance.
cudaError_t launch_pool_persistent(const PoolDevice& d, int tile, int steps, int blocks, cudaStream_t stream);
int pool_persistent_max_blocks(int tile);
// The tiled schedule (tiles of 128 tets): per element tile, its distinct nodes'
// displacements are gathered once into shared memory, each tet's corner forces are
// summed per node inside the tile (in tet order), and one partial per (tile, node) is
// written; the node pass sums a node's partials in ascending tile order.
//
// Building the tables for the current work list (d.etiles), in two passes over the
// tiles with the caller's exclusive scan of the spans into `off` between them (and the
// arrays sized for the total); the partial slots and part_off are then the node ->
// (tile, node) CSR of node_tab (build_csr_device).
// Pass 1 sorts each tile's corners and writes `count` (distinct nodes), `span` (that,
// padded to a multiple of 8: what `off` scans), `lidx` and `inv`.  Pass 2, with d.lidx
// set, writes node_tab and inv_start at the scanned offsets; the padding entries name
// node `dump`, one past every mesh's nodes.
void launch_pool_tile_count(const PoolDevice& d, uint32_t* count, uint32_t* span, ushort4* lidx, uint16_t* inv,
                            cudaStream_t stream);
void launch_pool_tile_fill(const PoolDevice& d, const uint32_t* off, const uint32_t* count, uint32_t* node_tab,
                           uint16_t* inv_start, uint32_t dump, cudaStream_t stream);
// The element pass of the tiled schedule: a persistent grid of blocks of 128 threads,
// each walking its tiles with the next tile's node gather and tables in flight; its
// node pass is launch_pool_node_pass over part_off and the partials.
void launch_pool_tiled_element_pass(const PoolDevice& d, int sub, cudaStream_t stream);

// One-time set-up of the pool's kernels on the current device (the staged pass's
// shared-memory size and grid); call outside any stream capture.
void pool_kernels_setup();
// meshes[id].dt = safety * 2 / sqrt(max omega^2) of the mesh's tets [t0, t0 + T),
// from the pool's FP32 Dm^-1; 0 when the bound is not positive.  `block_max` holds
// ceil(T / 256) doubles and `w2` one double of scratch.
// One mesh of an admission group, for the group's batched admission kernels: its
// ranges in the pool, where its tets / nodes / partial slots start among the group's
// (prefix sums, ascending), its density and elastic constants, and whether its time
// step is to be formed on the device.
struct PoolAdmit {
    long long t0, T, n0, N, part0, parts;
    long long tet_first, node_first, part_first;  // node_first counts N + 1 per mesh
    double density, lambda, mu;
    int id, want_dt;
};

// The device half of admitting a group of meshes, after their index, slot map, CSR
// offsets, pins, load, record and rest positions (staged in the velocity rows) are
// uploaded: zero the plastic state and the energy partials, form the FP64 rest state
// (Dm^-1, volumes, lumped masses), start the nodes at rest, and, for the meshes that
// want it, set the time step to 0.9 x the FP64 element bound, 2 / sqrt(max omega^2)
// over its tets (tet_omega2_one, the single-mesh handle's bound, normalising its iterate
// by a reciprocal: within rounding of the single-mesh value).
// `adm` (device) holds the G records; `w2` is G scratch words.  Four launches per
// group, whatever its size.
void launch_pool_admit(const PoolDevice& d, const PoolAdmit* adm, int G, long long tets, long long nodes,
                       long long parts, bool any_dt, unsigned long long* w2, cudaStream_t stream);
// index[0 .. tets) += (add, add, add, add): node ids of a group uploaded local to its
// span, rebased into the pool after the group's CSR was built from them.
void launch_pool_rebase(uint4* index, long long tets, uint32_t add, cudaStream_t stream);

}  // namespace fs
