// pool_tiled.cu -- the pool's tiled schedule: per-tile node gathers and per-(tile, node)
// force partials.
//
// In the other schedules every tet writes its four corner forces to node-major slots
// (64 B per tet) and the node pass reads them back (64 B per tet): half of a step's
// HBM traffic.  Here a block takes one element tile (up to 128 consecutive tets of one
// mesh) and:
//   1. gathers the displacements (and compensations) of the tile's distinct nodes once
//      into shared memory -- about 90 nodes for the 512 corners of a Kuhn box mesh;
//   2. evaluates each tet from its corners there, with the arithmetic of every other
//      schedule (tet_element_f32_eval), its corner forces into shared memory;
//   3. sums, for each distinct node, the corner forces of the tile's tets that name
//      it, in ascending tet order, and writes that one partial to the node's run of
//      the per-(tile, node) CSR;
// and the node pass sums a node's partials in ascending tile order (the other
// schedules' node kernel over this CSR).  Per tet, the slot traffic falls from 128 B to
// twice 16 B per (tile, node) pair -- about 22 B.
//
// A node's force is then (partial of its first tile) + (partial of the next) + ...,
// each partial summed in tet order: the same terms as the other schedules' single
// ascending run, associated per tile.  Tiles are aligned to their mesh's first tet, so
// the association, and with it every bit of a mesh's result, does not depend on where
// the mesh sits in the pool or what else is there; it differs from the other
// schedules' in rounding only.
//
// The tables are built on the device for each work list: per tile, its corners are
// sorted by (node, corner) in shared memory (a bitonic sort of 512 keys), which gives
// the distinct nodes in ascending order, each corner's place in that list and, per
// node, its corners in ascending order.
#include <algorithm>
#include <mutex>

#include <cub/block/block_scan.cuh>

#include "common.cuh"
#include "pool.hpp"
#include "tet_f32.cuh"

namespace fs {
namespace {

constexpr int kTiledTile = 128;              // tets per tile
constexpr int kTiledCorners = 4 * kTiledTile;  // 512

// The tile's corners, sorted: key = node << 9 | corner (corner = 4 x tet-in-tile + c);
// slots past the tile's corners hold ~0 and sort last.  All 128 threads call it.
__device__ __forceinline__ void sort_tile_corners(const PoolDevice& d, const PoolTile& tl,
                                                  unsigned long long* key) {
    const int corners = 4 * (int)(tl.end - tl.begin);
    for (int i = threadIdx.x; i < kTiledCorners; i += kTiledTile) {
        unsigned long long k = ~0ull;
        if (i < corners) {
            const uint4 id = d.index[tl.begin + (i >> 2)];
            const uint32_t c = i & 3;
            const uint32_t node = c == 0 ? id.x : (c == 1 ? id.y : (c == 2 ? id.z : id.w));
            k = ((unsigned long long)node << 9) | (unsigned long long)i;
        }
        key[i] = k;
    }
    __syncthreads();
    for (int size = 2; size <= kTiledCorners; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = threadIdx.x; i < kTiledCorners; i += kTiledTile) {
                const int j = i ^ stride;
                if (j > i) {
                    const unsigned long long a = key[i], b = key[j];
                    const bool up = (i & size) == 0;
                    if ((a > b) == up) {
                        key[i] = b;
                        key[j] = a;
                    }
                }
            }
            __syncthreads();
        }
}

// The sorted position i starts a new node (and is a real corner).
__device__ __forceinline__ bool starts_node(const unsigned long long* key, int i) {
    if (key[i] == ~0ull) return false;
    return i == 0 || (key[i] >> 9) != (key[i - 1] >> 9);
}

using TileScan = cub::BlockScan<int, kTiledTile>;

// Each thread takes four consecutive sorted positions; returns the thread's exclusive
// prefix of node starts, and the tile's total in `total`.
__device__ __forceinline__ int scan_node_starts(const unsigned long long* key, int (&flag)[4], int& total,
                                                typename TileScan::TempStorage& tmp) {
    int mine = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        flag[q] = starts_node(key, 4 * threadIdx.x + q) ? 1 : 0;
        mine += flag[q];
    }
    int before = 0;
    TileScan(tmp).ExclusiveSum(mine, before, total);
    return before;
}

// A tile's lists are padded to a multiple of 8 entries, so each starts on a 16-byte
// boundary (for the staged pass's asynchronous copies).
constexpr int kTablePad = 8;

// Pass 1: per tile, its corners sorted; the distinct-node count (and its padded
// span), and the two tables that need no global offset: the sorted corners (inv) and
// each tet's corner places in the tile's node list (lidx).
__global__ void __launch_bounds__(kTiledTile) pool_tile_count(PoolDevice d, uint32_t* count, uint32_t* span,
                                                               ushort4* lidx, uint16_t* inv) {
    __shared__ unsigned long long key[kTiledCorners];
    __shared__ uint16_t local[kTiledCorners];  // by corner: its node's place in the list
    __shared__ typename TileScan::TempStorage tmp;
    const PoolTile tl = d.etiles[blockIdx.x];
    sort_tile_corners(d, tl, key);
    int flag[4], total = 0;
    int at = scan_node_starts(key, flag, total, tmp) - 1;  // the node of position 4 x thread - 1
    const long long c0 = 4 * tl.begin;  // the tile's corners in the per-corner arrays
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int i = 4 * threadIdx.x + q;
        const unsigned long long k = key[i];
        if (k == ~0ull) continue;
        if (flag[q]) ++at;
        const int corner = (int)(k & 511ull);
        // stored as the corner's place in the element pass's force buffer, corner c of
        // tet i at c x 128 + i
        inv[c0 + i] = (uint16_t)((corner & 3) * kTiledTile + (corner >> 2));
        local[corner] = (uint16_t)at;
    }
    if (threadIdx.x == 0) {
        count[blockIdx.x] = (uint32_t)total;
        span[blockIdx.x] = (uint32_t)((total + kTablePad - 1) / kTablePad * kTablePad);
    }
    __syncthreads();
    const long long t = tl.begin + threadIdx.x;
    if (t < tl.end) {
        const int c = 4 * threadIdx.x;
        lidx[t] = make_ushort4(local[c], local[c + 1], local[c + 2], local[c + 3]);
    }
}

// Pass 2, after the scan of the spans into `off`: the node list and, per node, the
// start of its corners in the sorted list -- from the corner places alone, without a
// second sort: a node's start is the number of the tile's corners whose nodes come
// before it in the list.  Padding entries name node `dump`, one past every mesh's
// nodes, so that the partials' CSR counts them under a node no tile reads.
__global__ void __launch_bounds__(kTiledTile) pool_tile_fill(PoolDevice d, const uint32_t* off, const uint32_t* count,
                                                              uint32_t* node_tab, uint16_t* inv_start,
                                                              uint32_t dump) {
    __shared__ int hist[kTiledCorners];
    __shared__ typename TileScan::TempStorage tmp;
    const PoolTile tl = d.etiles[blockIdx.x];
    const uint32_t base = off[blockIdx.x];
    const int total = (int)count[blockIdx.x];
    for (int j = threadIdx.x; j < kTiledCorners; j += kTiledTile) hist[j] = 0;
    __syncthreads();
    const long long t = tl.begin + threadIdx.x;
    if (t < tl.end) {
        const ushort4 l = d.lidx[t];
        const uint4 id = d.index[t];
        atomicAdd(&hist[l.x], 1);
        atomicAdd(&hist[l.y], 1);
        atomicAdd(&hist[l.z], 1);
        atomicAdd(&hist[l.w], 1);
        // every corner of a node writes the same id
        node_tab[base + l.x] = id.x;
        node_tab[base + l.y] = id.y;
        node_tab[base + l.z] = id.z;
        node_tab[base + l.w] = id.w;
    }
    __syncthreads();
    // exclusive scan of the per-node corner counts: four consecutive nodes a thread
    int v[4], mine = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        v[q] = hist[4 * threadIdx.x + q];
        mine += v[q];
    }
    int before = 0, all = 0;
    TileScan(tmp).ExclusiveSum(mine, before, all);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int j = 4 * threadIdx.x + q;
        if (j < total) inv_start[base + j] = (uint16_t)before;
        before += v[q];
    }
    const int padded = (total + kTablePad - 1) / kTablePad * kTablePad;
    if ((int)threadIdx.x < padded - total) {
        node_tab[base + total + threadIdx.x] = dump;
        inv_start[base + total + threadIdx.x] = 0;
    }
}

// Dm^-1 (9 rows), the volume and the plastic state (7 rows)
constexpr int kRowsPrefetched = 17;

// L2 prefetch, by one warp (lane 0..31, a few lines each), of the rows the tiled pass
// reads for tets [begin, end): the corner places (8 B per tet), Dm^-1 (9 rows of 4 B),
// the volume and the plastic state (7 rows); every line starts inside its row's range.
__device__ __forceinline__ void prefetch_tiled_rows_warp(const PoolDevice& d, long long begin, long long end,
                                                         int lane) {
    if (end <= begin) return;
    const long long n = end - begin;
    const int wide = (int)((n * 8 + 127) >> 7);
    const int narrow = (int)((n * 4 + 127) >> 7);
    for (int k = lane; k < wide; k += 32)
        prefetch_l2(reinterpret_cast<const char*>(d.lidx + begin) + ((long long)k << 7));
    for (int k = lane; k < kRowsPrefetched * narrow; k += 32) {
        const int row = k / narrow, line = k - row * narrow;
        const float* rowp = row < 9 ? d.rest_inv + (size_t)row * d.tet_cap
                                    : (row == 9 ? d.rest_vol : d.plastic + (size_t)(row - 10) * d.tet_cap);
        prefetch_l2(reinterpret_cast<const char*>(rowp + begin) + ((long long)line << 7));
    }
}

// A tet's own rows, loaded into registers before the tile's corners arrive (so their
// latency runs alongside the wait), handed to tet_element_f32_eval as its `Rows`.
struct RegRows {
    float dm[9], v, pl[7];
    __device__ __forceinline__ float inv(int k, long long) const { return dm[k]; }
    __device__ __forceinline__ float vol(long long) const { return v; }
    __device__ __forceinline__ float plastic(int i, long long) const { return pl[i]; }
};

// ---- the staged form: a persistent block walks its tiles, and while it computes one,
// the next one's node gather and tables are already on their way into the other of two
// shared-memory stages (cp.async, per thread, completed by wait_group and a barrier).

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// One stage for tiles of up to `kcap` distinct nodes (a multiple of 8): the nodes'
// displacement and compensation, the tile's corner starts and partial slots (padded
// lists, copied whole), its corners sorted by node.
struct TiledStage {
    float4* su;
    float4* sc;
    uint32_t* slot;
    uint16_t* start;
    uint16_t* inv;
    __device__ __forceinline__ TiledStage(unsigned char* p, int kcap) {
        su = reinterpret_cast<float4*>(p);
        sc = su + kcap;
        slot = reinterpret_cast<uint32_t*>(sc + kcap);
        start = reinterpret_cast<uint16_t*>(slot + kcap);
        inv = start + kcap;
    }
    __host__ __device__ static size_t bytes(int kcap) {
        return (size_t)kcap * 32 + (size_t)kcap * 4 + (size_t)kcap * 2 + (size_t)kTiledCorners * 2;
    }
};

// What a block needs of its tile, kept in shared memory by the fill that loaded it.
struct TiledInfo {
    long long begin, end;
    uint32_t base;
    int k, mesh, part, live;
};

// Queue the copies of tile g's gather and tables into `st` (every thread its share);
// thread 0 records the tile in `info`.
__device__ __forceinline__ void tiled_fill(const PoolDevice& d, int g, int sub, const TiledStage& st,
                                           TiledInfo& info) {
    const PoolTile tl = d.etiles[g];
    const PoolMesh& m = d.meshes[tl.mesh];
    const bool live = m.step + sub < m.target;
    const uint32_t base = d.tab_off[g];
    const int k = (int)d.tab_count[g];
    if (threadIdx.x == 0) info = TiledInfo{tl.begin, tl.end, base, k, tl.mesh, tl.part, live ? 1 : 0};
    if (!live) return;  // a frozen mesh's tile reads nothing
    const int kp = (k + kTablePad - 1) / kTablePad * kTablePad;
    for (int j = threadIdx.x; j < k; j += kTiledTile) {
        const uint32_t n = d.node_tab[base + j];
        cp_async16(st.su + j, d.disp + n);
        cp_async16(st.sc + j, d.disp_c + n);
    }
    // the padded lists from their 16-byte aligned starts: 4 slots, or 8 starts, a copy
    for (int q = threadIdx.x; q < kp / 4; q += kTiledTile) cp_async16(st.slot + 4 * q, d.part_slot + base + 4 * q);
    for (int q = threadIdx.x; q < kp / 8; q += kTiledTile)
        cp_async16(st.start + 8 * q, d.inv_start + base + 8 * q);
    // the sorted corners: four of them (8 bytes) per tet
    const int n = (int)(tl.end - tl.begin);
    if ((int)threadIdx.x < n) cp_async8(st.inv + 4 * threadIdx.x, d.inv + 4 * (tl.begin + threadIdx.x));
}

__global__ void __launch_bounds__(kTiledTile, 1024 / kTiledTile) pool_elements_tiled_ring(PoolDevice d, int sub,
                                                                                          int kcap) {
    extern __shared__ __align__(16) unsigned char tiled_smem[];
    __shared__ float4 sf[kTiledCorners];  // corner c of tet i at c x 128 + i
    __shared__ double scratch[64];
    __shared__ TiledInfo info[2];
    const int G = (int)gridDim.x;
    int g = blockIdx.x;
    if (g >= d.n_etiles) return;
    const TiledStage st0(tiled_smem, kcap), st1(tiled_smem + TiledStage::bytes(kcap), kcap);
    tiled_fill(d, g, sub, st0, info[0]);
    cp_async_commit();
    for (int it = 0;; ++it) {
        const TiledStage& cur = (it & 1) ? st1 : st0;
        const TiledStage& oth = (it & 1) ? st0 : st1;
        const int nxt = g + G;
        // the tile after next into L2, its rows and tables, by the last warp alone
        if (threadIdx.x >= kTiledTile - 32 && nxt + G < d.n_etiles) {
            const PoolTile nx = d.etiles[nxt + G];
            const int lane = threadIdx.x - (kTiledTile - 32);
            prefetch_tiled_rows_warp(d, nx.begin, nx.end, lane);
            const uint32_t ob = d.tab_off[nxt + G];
            if (lane == 0) prefetch_l2(d.node_tab + ob);
            if (lane == 1) prefetch_l2(d.part_slot + ob);
            if (lane == 2) prefetch_l2(d.inv_start + ob);
        }
        // this tile, as its fill recorded it: visible after the barriers of the tile before
        // (its wait), or, for the first tile, after this one
        if (it == 0) __syncthreads();
        const TiledInfo& ti = info[it & 1];
        const PoolMesh& m = d.meshes[ti.mesh];
        const bool live = ti.live != 0;
        const long long t = ti.begin + threadIdx.x;
        const bool mine = live && t < ti.end;
        // this tet's rows and corner places into registers (their latency overlaps the wait)
        RegRows rr;
        ushort4 l = make_ushort4(0, 0, 0, 0);
        if (mine) {
            l = d.lidx[t];
#pragma unroll
            for (int q = 0; q < 9; ++q) rr.dm[q] = d.rest_inv[(size_t)q * d.tet_cap + t];
            rr.v = d.rest_vol[t];
#pragma unroll
            for (int i = 0; i < 7; ++i) rr.pl[i] = d.plastic[(size_t)i * d.tet_cap + t];
        }
        // the next tile's copies go out now; this tile's have landed once all but the
        // newest group are done, in every thread
        if (nxt < d.n_etiles) tiled_fill(d, nxt, sub, oth, info[(it & 1) ^ 1]);
        cp_async_commit();
        cp_async_wait_one();
        __syncthreads();
        double diss = 0.0, energy = 0.0;
        if (mine) {
            const float4 un[4] = {cur.su[l.x], cur.su[l.y], cur.su[l.z], cur.su[l.w]};
            const float4 cn[4] = {cur.sc[l.x], cur.sc[l.y], cur.sc[l.z], cur.sc[l.w]};
            const TetElementRefs r{d.index,     d.slot, d.rest_inv, d.rest_vol, d.plastic,
                                   d.plastic_c, d.disp, d.disp_c,   d.slots,    d.tet_cap};
            float4 fc[4];
            tet_element_f32_eval<true, RegRows>(r, rr, t, m.mat, un, cn, diss, energy, fc);
            sf[threadIdx.x] = fc[0];
            sf[kTiledTile + threadIdx.x] = fc[1];
            sf[2 * kTiledTile + threadIdx.x] = fc[2];
            sf[3 * kTiledTile + threadIdx.x] = fc[3];
        }
        __syncthreads();
        if (live) {
            const int k = ti.k;
            const int corners = 4 * (int)(ti.end - ti.begin);
            for (int j = threadIdx.x; j < k; j += kTiledTile) {
                const int b = cur.start[j], e = j + 1 < k ? cur.start[j + 1] : corners;
                float4 f = sf[cur.inv[b]];
                for (int q = b + 1; q < e; ++q) {
                    const float4 h = sf[cur.inv[q]];
                    f.x += h.x;
                    f.y += h.y;
                    f.z += h.z;
                }
                d.slots[cur.slot[j]] = make_float4(f.x, f.y, f.z, 0.0f);
            }
        }
        block_sum2(diss, energy, scratch);  // valid in thread 0; also ends the stage's reads
        if (live && threadIdx.x == 0) {
            d.e_diss[ti.part] += diss;
            d.e_strain[ti.part] = energy;
        }
        if (nxt >= d.n_etiles) break;
        g = nxt;
    }
    cp_async_wait_all();
}

}  // namespace

void launch_pool_tiled_element_pass(const PoolDevice& d, int sub, cudaStream_t stream) {
    if (!d.n_etiles || d.tab_kcap <= 0) return;  // no tables: nothing to step
    // a persistent grid of as many blocks as fit with two stages of kcap nodes.  The
    // kernel's dynamic shared-memory ceiling only ever grows (under a lock), so a pool
    // with smaller stages, in this thread or another, never lowers it under a launch.
    static std::mutex lock;
    static size_t ceiling = 0;
    const size_t dyn = 2 * TiledStage::bytes(d.tab_kcap);
    int per_sm = 0;
    {
        std::lock_guard<std::mutex> hold(lock);
        if (dyn > ceiling) {
            cudaFuncSetAttribute(pool_elements_tiled_ring, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
            ceiling = dyn;
        }
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pool_elements_tiled_ring, kTiledTile, dyn);
    }
    const int grid = std::min(d.n_etiles, std::max(per_sm, 1) * sm_count());
    pool_elements_tiled_ring<<<grid, kTiledTile, dyn, stream>>>(d, sub, d.tab_kcap);
}

void launch_pool_tile_count(const PoolDevice& d, uint32_t* count, uint32_t* span, ushort4* lidx, uint16_t* inv,
                            cudaStream_t stream) {
    if (d.n_etiles) pool_tile_count<<<d.n_etiles, kTiledTile, 0, stream>>>(d, count, span, lidx, inv);
}

void launch_pool_tile_fill(const PoolDevice& d, const uint32_t* off, const uint32_t* count, uint32_t* node_tab,
                           uint16_t* inv_start, uint32_t dump, cudaStream_t stream) {
    if (d.n_etiles)
        pool_tile_fill<<<d.n_etiles, kTiledTile, 0, stream>>>(d, off, count, node_tab, inv_start, dump);
}

}  // namespace fs
