// api_pool.cu -- host side of the multi-mesh pool (pool.hpp) behind the C ABI.
//
// The pool is the engine of both the batched and the served workloads: meshes are
// admitted into free ranges of the pool's arrays against its capacity, stepped
// together (each with its own material, load, time step and step count), read back
// and released.  Admission that does not fit returns FEMSTEP_ENOMEM, so a serving
// loop keeps the request queued and admits it as soon as a release frees room; the
// requests already on the GPU keep running meanwhile (continuous batching).
//
// Everything the pool does on the device goes through its one stream, in call order.
// That makes every call safe while a chunk is still running: an admission's uploads,
// a release's freeze and a new work list all land behind the chunk.  Admission does
// its host work (rest state, CSR, slot map) while the GPU runs and hands the bytes to
// the stream from pinned staging buffers, so it never waits for the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <string>
#include <mutex>
#include <thread>
#include <vector>

#include <cub/device/device_reduce.cuh>
#include <cub/device/device_scan.cuh>

#include "../../include/femstep.h"
#include "common.cuh"
#include "host_util.hpp"
#include "pool.hpp"
#include "shell.hpp"
#include "tet.hpp"

using fs::PoolDevice;
using fs::PoolMesh;
using fs::PoolTile;

namespace {

// First-fit allocator over [0, capacity) with coalescing on release.
class RangeAllocator {
public:
    void reset(long long capacity) {
        free_.clear();
        if (capacity > 0) free_[0] = capacity;
    }
    long long take(long long n) {
        for (auto it = free_.begin(); it != free_.end(); ++it)
            if (it->second >= n) {
                const long long at = it->first, left = it->second - n;
                free_.erase(it);
                if (left > 0) free_[at + n] = left;
                return at;
            }
        return -1;
    }
    void give(long long at, long long n) {
        auto next = free_.lower_bound(at);
        if (next != free_.end() && at + n == next->first) {
            n += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == at) {
                prev->second += n;
                return;
            }
        }
        free_[at] = n;
    }

private:
    std::map<long long, long long> free_;  // start -> length
};

// Pinned host memory outlives the pools that staged through it: pinning is the slow
// part of getting it (tens of milliseconds per 64 MB), so a destroyed pool hands its
// buffers to this process-wide cache, up to kHostCacheBytes, and the next pool takes
// them from here before it pins anything new.  Buffers are portable (usable from any
// device of the process); the memory returns to the system when the process exits.
class HostCache {
public:
    static HostCache& get() {
        static HostCache* cache = new HostCache();  // never destroyed: no CUDA calls at exit
        return *cache;
    }
    // The smallest cached buffer of at least `bytes`, or null.
    char* take(size_t bytes, size_t& cap) {
        std::lock_guard<std::mutex> lock(mu_);
        auto it = free_.lower_bound(bytes);
        if (it == free_.end()) return nullptr;
        cap = it->first;
        char* p = it->second;
        total_ -= cap;
        free_.erase(it);
        return p;
    }
    // Keep `p` for a later pool, or free it when the cache is full.
    void give(char* p, size_t cap) {
        {
            std::lock_guard<std::mutex> lock(mu_);
            if (total_ + cap <= kHostCacheBytes) {
                free_.emplace(cap, p);
                total_ += cap;
                return;
            }
        }
        cudaFreeHost(p);
    }

private:
    static constexpr size_t kHostCacheBytes = size_t(1) << 30;
    std::mutex mu_;
    std::multimap<size_t, char*> free_;
    size_t total_ = 0;
};

// Pinned host buffers for uploads queued behind device work.  A buffer is reused once
// the event recorded after its copies has completed.
class Staging {
public:
    struct Buf {
        char* host = nullptr;
        size_t cap = 0, used = 0;
        cudaEvent_t done = nullptr;
        bool pending = false;
    };
    // A buffer of at least `bytes`, not in use by any queued copy.
    Buf* get(size_t bytes, cudaError_t& err) {
        err = cudaSuccess;
        Buf* best = nullptr;
        for (Buf& b : bufs_) {
            if (b.pending) {
                if (cudaEventQuery(b.done) != cudaSuccess) continue;
                b.pending = false;
            }
            if (b.cap >= bytes && (!best || b.cap < best->cap)) best = &b;
        }
        if (!best) {
            // capacities are powers of two (at least 4 MB), so buffers of one size class
            // serve every later request of that class: a few buffers, reused -- and kept
            // across pools by the host cache
            Buf b;
            b.cap = size_t(4) << 20;
            while (b.cap < bytes) b.cap <<= 1;
            size_t cached = 0;
            b.host = HostCache::get().take(b.cap, cached);
            if (b.host) {
                b.cap = cached;
            } else {
                err = cudaHostAlloc(&b.host, b.cap, cudaHostAllocPortable);
                if (err != cudaSuccess) return nullptr;
            }
            err = cudaEventCreateWithFlags(&b.done, cudaEventDisableTiming);
            if (err != cudaSuccess) {
                HostCache::get().give(b.host, b.cap);
                return nullptr;
            }
            bufs_.push_back(b);
            best = &bufs_.back();
        }
        best->used = 0;
        return best;
    }
    // Reserve `bytes` (256-aligned) inside `b`.
    static char* take(Buf* b, size_t bytes) {
        char* p = b->host + b->used;
        b->used += (bytes + 255) & ~size_t(255);
        return p;
    }
    static void submit(Buf* b, cudaStream_t s) {
        cudaEventRecord(b->done, s);
        b->pending = true;
    }
    // After the pool's stream has drained: the buffers go to the host cache.
    void release() {
        for (Buf& b : bufs_) {
            if (b.done) cudaEventDestroy(b.done);
            if (b.host) HostCache::get().give(b.host, b.cap);
        }
        bufs_.clear();
    }
    size_t count() const { return bufs_.size(); }

private:
    std::deque<Buf> bufs_;  // a deque, so a Buf* stays valid as buffers are added
};

struct HostMesh {
    bool used = false;
    long long t0 = 0, T = 0, n0 = 0, N = 0;  // pool ranges (N + 1 node slots held)
    long long e_part = 0, n_part = 0, e_tiles = 0, n_tiles = 0;  // partial slots (tile 128)
    long long target = 0, serial = 0;
    std::vector<float> rest;                  // 3N rest positions, for readback
};

constexpr int kMinTile = 128;
constexpr int kGraphSteps = 16;

}  // namespace

struct femstep_pool {
    long long tet_cap = 0, node_cap = 0, part_cap = 0;
    int max_meshes = 0;
    long long next_serial = 1;
    int tile = 256;
    int mode = FEMSTEP_POOL_GRAPH;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    fs::DeviceArena arena;
    PoolDevice d;
    RangeAllocator tets, nodes, parts;
    std::vector<HostMesh> meshes;
    Staging staging;
    bool dirty = true;  // work lists need rebuilding
    PoolTile* d_etiles = nullptr;
    PoolTile* d_ntiles = nullptr;
    int* d_active = nullptr;
    fs::PoolAdmit* d_admit = nullptr;  // [max_meshes]: an admission group's records
    unsigned long long* d_w2 = nullptr;  // [max_meshes]: the group's element bounds
    cudaGraphExec_t graph = nullptr;
    fs::PoolPasses graph_passes = fs::PoolPasses::kDirect;  // what the graph was captured with
    // the tiled schedule's tables for the current work list, allocated at first use
    struct Tiled {
        bool valid = false;
        uint32_t *count = nullptr, *span = nullptr, *off = nullptr, *part_off = nullptr, *kmax = nullptr;
        ushort4* lidx = nullptr;
        uint16_t* inv = nullptr;
        uint32_t *node_tab = nullptr, *part_slot = nullptr;
        uint16_t* inv_start = nullptr;
        size_t entries_cap = 0;
        size_t fixed_bytes = 0;       // the per-capacity arrays, allocated at first use
        void* scan_tmp = nullptr;
        size_t scan_bytes = 0;
        uint32_t* h_total = nullptr;  // pinned: [0] last tile's offset, [1] its span, [2] the largest count
        int max_nodes = 0;            // distinct nodes of the largest tile
    } tiled;
    long long launches = 0;
    bool in_flight = false;
    bool broken = false;
    double* d_out = nullptr;
    PoolMesh* h_meshes = nullptr;  // pinned mirror of the mesh table, refreshed per chunk
    int* h_error = nullptr;        // pinned mirror of the barrier error flag
    std::string error;
};

namespace {

int fail(femstep_pool* p, int code, const std::string& what) {
    if (p) p->error = what;
    fs::set_last_error(what);
    return code;
}

int check(femstep_pool* p, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return FEMSTEP_OK;
    return fail(p, e == cudaErrorMemoryAllocation ? FEMSTEP_ENOMEM : FEMSTEP_ECUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

bool valid_mode(int mode) {
    return mode == FEMSTEP_POOL_GRAPH || mode == FEMSTEP_POOL_PERSISTENT || mode == FEMSTEP_POOL_GRAPH_STAGED ||
           mode == FEMSTEP_POOL_GRAPH_TILED;
}

bool valid_id(const femstep_pool* p, int id) { return p && id >= 0 && id < p->max_meshes && p->meshes[id].used; }

void drop_graph(femstep_pool* p) {
    if (p->graph) cudaGraphExecDestroy(p->graph);
    p->graph = nullptr;
}

// Rebuild the tile lists of the admitted meshes (tiles never straddle meshes) and
// queue their upload; the lists' device buffers are sized for the pool's capacity.
int rebuild(femstep_pool* p) {
    if (!p->dirty) return FEMSTEP_OK;
    std::vector<PoolTile> et, nt;
    std::vector<int> active;
    const int T = p->tile;
    for (int id = 0; id < (int)p->meshes.size(); ++id) {
        const HostMesh& m = p->meshes[id];
        if (!m.used) continue;
        active.push_back(id);
        for (long long k = 0, b = 0; b < m.T; ++k, b += T)
            et.push_back(PoolTile{id, (int)(m.e_part + k), m.t0 + b, m.t0 + std::min(m.T, b + T)});
        for (long long k = 0, b = 0; b < m.N; ++k, b += T)
            nt.push_back(PoolTile{id, (int)(m.n_part + k), m.n0 + b, m.n0 + std::min(m.N, b + T)});
    }
    if ((long long)et.size() > p->part_cap || (long long)nt.size() > p->part_cap)
        return fail(p, FEMSTEP_ESTATE, "work list above its capacity");
    const size_t be = et.size() * sizeof(PoolTile), bn = nt.size() * sizeof(PoolTile),
                 ba = active.size() * sizeof(int);
    cudaError_t err;
    Staging::Buf* buf = p->staging.get(be + bn + ba + 3 * 256, err);
    if (!buf) return check(p, err, "pinned staging");
    auto put = [&](void* dst, const void* src, size_t bytes) {
        if (!bytes) return;
        char* h = Staging::take(buf, bytes);
        std::memcpy(h, src, bytes);
        cudaMemcpyAsync(dst, h, bytes, cudaMemcpyHostToDevice, p->stream);
    };
    put(p->d_etiles, et.data(), be);
    put(p->d_ntiles, nt.data(), bn);
    put(p->d_active, active.data(), ba);
    Staging::submit(buf, p->stream);
    p->d.etiles = p->d_etiles;
    p->d.ntiles = p->d_ntiles;
    p->d.n_etiles = (int)et.size();
    p->d.n_ntiles = (int)nt.size();
    p->d.active = p->d_active;
    p->d.n_active = (int)active.size();
    p->dirty = false;
    p->tiled.valid = false;
    drop_graph(p);
    return check(p, cudaGetLastError(), "work list upload");
}

fs::PoolPasses passes_of(int mode) {
    return mode == FEMSTEP_POOL_GRAPH_STAGED  ? fs::PoolPasses::kStaged
           : mode == FEMSTEP_POOL_GRAPH_TILED ? fs::PoolPasses::kTiled
                                              : fs::PoolPasses::kDirect;
}

void free_tiled(femstep_pool* p) {
    auto& t = p->tiled;
    for (void* q : {(void*)t.count, (void*)t.span, (void*)t.off, (void*)t.part_off, (void*)t.kmax, (void*)t.lidx,
                    (void*)t.inv, (void*)t.node_tab, (void*)t.part_slot, (void*)t.inv_start, t.scan_tmp})
        fs::device_free(q);
    if (t.h_total) cudaFreeHost(t.h_total);
    t = femstep_pool::Tiled{};
}

// The tiled schedule's tables for the current work list (tiles of 128): per tile its
// distinct nodes, counted, scanned and filled on the device, then the node -> (tile,
// node) CSR of the partials.  Waits once for the total count, to size the per-entry
// arrays.
int ensure_tiled(femstep_pool* p) {
    auto& t = p->tiled;
    if (t.valid) return FEMSTEP_OK;
    if (p->tile != 128) return fail(p, FEMSTEP_EINVAL, "the tiled schedule runs tiles of 128");
    PoolDevice& d = p->d;
    const int G = d.n_etiles;
    if (G == 0) return FEMSTEP_OK;
    cudaError_t e = cudaSuccess;
    if (!t.count) {
        e = fs::device_alloc((void**)&t.count, (size_t)p->part_cap * 4);
        if (e == cudaSuccess) e = fs::device_alloc((void**)&t.span, (size_t)p->part_cap * 4);
        if (e == cudaSuccess) e = fs::device_alloc((void**)&t.off, (size_t)p->part_cap * 4);
        if (e == cudaSuccess) e = fs::device_alloc((void**)&t.kmax, 4);
        if (e == cudaSuccess) e = fs::device_alloc((void**)&t.part_off, (size_t)(p->node_cap + 2) * 4);
        if (e == cudaSuccess) e = fs::device_alloc((void**)&t.lidx, (size_t)p->tet_cap * sizeof(ushort4));
        if (e == cudaSuccess) e = fs::device_alloc((void**)&t.inv, (size_t)p->tet_cap * 4 * sizeof(uint16_t));
        t.fixed_bytes = (size_t)p->part_cap * 12 + 4 + (size_t)(p->node_cap + 2) * 4 + (size_t)p->tet_cap * 16;
        size_t reduce_bytes = 0;
        if (e == cudaSuccess)
            e = cub::DeviceScan::ExclusiveSum(nullptr, t.scan_bytes, t.span, t.off, (int)p->part_cap, p->stream);
        if (e == cudaSuccess)
            e = cub::DeviceReduce::Max(nullptr, reduce_bytes, t.count, t.kmax, (int)p->part_cap, p->stream);
        t.scan_bytes = std::max(t.scan_bytes, reduce_bytes);
        if (e == cudaSuccess) e = fs::device_alloc(&t.scan_tmp, t.scan_bytes ? t.scan_bytes : 1);
        if (e == cudaSuccess) e = cudaHostAlloc((void**)&t.h_total, 3 * sizeof(uint32_t), cudaHostAllocPortable);
        if (e != cudaSuccess) {
            free_tiled(p);
            return check(p, e, "tiled tables");
        }
    }
    fs::launch_pool_tile_count(d, t.count, t.span, t.lidx, t.inv, p->stream);
    size_t tmp_bytes = t.scan_bytes;
    e = cub::DeviceScan::ExclusiveSum(t.scan_tmp, tmp_bytes, t.span, t.off, G, p->stream);
    tmp_bytes = t.scan_bytes;
    if (e == cudaSuccess) e = cub::DeviceReduce::Max(t.scan_tmp, tmp_bytes, t.count, t.kmax, G, p->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(t.h_total, t.off + (G - 1), 4, cudaMemcpyDeviceToHost, p->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(t.h_total + 1, t.span + (G - 1), 4, cudaMemcpyDeviceToHost, p->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(t.h_total + 2, t.kmax, 4, cudaMemcpyDeviceToHost, p->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(p->stream);
    if (e != cudaSuccess) return check(p, e, "tiled tables");
    const size_t total = (size_t)t.h_total[0] + t.h_total[1];
    t.max_nodes = (int)t.h_total[2];
    if (total > t.entries_cap) {
        fs::device_free(t.node_tab);
        fs::device_free(t.part_slot);
        fs::device_free(t.inv_start);
        t.node_tab = t.part_slot = nullptr;
        t.inv_start = nullptr;
        const size_t cap = total + total / 4 + 1024;
        e = fs::device_alloc((void**)&t.node_tab, cap * 4);
        if (e == cudaSuccess) e = fs::device_alloc((void**)&t.part_slot, cap * 4);
        if (e == cudaSuccess) e = fs::device_alloc((void**)&t.inv_start, cap * 2);
        if (e != cudaSuccess) {
            t.entries_cap = 0;
            return check(p, e, "tiled tables");
        }
        t.entries_cap = cap;
    }
    long long nmax = 0;
    for (const HostMesh& m : p->meshes)
        if (m.used) nmax = std::max(nmax, m.n0 + m.N + 1);
    // the padding entries name node nmax, past every mesh, which the CSR leaves out
    d.lidx = t.lidx;
    d.inv = t.inv;
    fs::launch_pool_tile_fill(d, t.off, t.count, t.node_tab, t.inv_start, (uint32_t)nmax, p->stream);
    e = fs::build_csr_device(t.node_tab, (long long)total, nmax, t.part_off, t.part_slot, p->stream, nullptr, 0);
    if (e != cudaSuccess) return check(p, e, "tiled partial CSR");
    d.tab_off = t.off;
    d.tab_count = t.count;
    d.node_tab = t.node_tab;
    d.inv_start = t.inv_start;
    d.part_slot = t.part_slot;
    d.lidx = t.lidx;
    d.inv = t.inv;
    d.part_off = t.part_off;
    d.tab_kcap = std::max(8, (t.max_nodes + 7) / 8 * 8);
    t.valid = true;
    return check(p, cudaGetLastError(), "tiled tables");
}

// The graph of kGraphSteps steps over the current work list, captured once (nothing
// runs while it is captured).
int ensure_graph(femstep_pool* p, fs::PoolPasses passes) {
    if (p->graph && p->graph_passes != passes) drop_graph(p);
    if (passes == fs::PoolPasses::kTiled) {
        const int rc = ensure_tiled(p);
        if (rc) return rc;
    }
    if (p->graph) return FEMSTEP_OK;
    cudaGraph_t g = nullptr;
    int rc = check(p, cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal), "capture");
    if (rc) return rc;
    fs::launch_pool_steps(p->d, p->tile, kGraphSteps, p->stream, passes);
    rc = check(p, cudaStreamEndCapture(p->stream, &g), "capture end");
    if (rc) return rc;
    rc = check(p, cudaGraphInstantiate(&p->graph, g, 0), "graph instantiate");
    cudaGraphDestroy(g);
    if (rc) return rc;
    p->graph_passes = passes;
    return FEMSTEP_OK;
}

int launch_chunk(femstep_pool* p, int steps, int mode) {
    if (steps <= 0 || p->d.n_etiles == 0) return FEMSTEP_OK;
    if (mode == FEMSTEP_POOL_PERSISTENT) {
        const int blocks = std::min(fs::pool_persistent_max_blocks(p->tile), p->d.n_etiles);
        if (blocks <= 0) return fail(p, FEMSTEP_ECUDA, "no co-resident blocks for the persistent launch");
        const int rc = check(p, fs::launch_pool_persistent(p->d, p->tile, steps, blocks, p->stream),
                             "persistent launch");
        p->launches += 2;
        return rc;
    }
    const fs::PoolPasses passes = passes_of(mode);
    if (passes == fs::PoolPasses::kTiled) {
        const int rc = ensure_tiled(p);
        if (rc) return rc;
    }
    int left = steps;
    if (left >= kGraphSteps) {
        const int rc = ensure_graph(p, passes);
        if (rc) return rc;
        for (; left >= kGraphSteps; left -= kGraphSteps) {
            const int rc = check(p, cudaGraphLaunch(p->graph, p->stream), "graph launch");
            if (rc) return rc;
            p->launches += 2 * kGraphSteps + 1;
        }
    }
    if (left > 0) {
        fs::launch_pool_steps(p->d, p->tile, left, p->stream, passes);
        p->launches += 2 * left + 1;
    }
    return check(p, cudaGetLastError(), "kernel launch");
}

// Everything a step changes, over the used prefix of the pool: the state a trial run
// is rolled back to.
struct Snapshot {
    std::vector<std::pair<void*, size_t>> spans;
    char* buf = nullptr;
};

int snapshot(femstep_pool* p, Snapshot& s, bool restore) {
    long long tmax = 0, nmax = 0, pmax = 0;
    for (const HostMesh& m : p->meshes)
        if (m.used) {
            tmax = std::max(tmax, m.t0 + m.T);
            nmax = std::max(nmax, m.n0 + m.N + 1);
            pmax = std::max(pmax, std::max(m.e_part + m.e_tiles, m.n_part + m.n_tiles));
        }
    if (!restore) {
        s.spans.clear();
        for (int k = 0; k < 7; ++k) {
            s.spans.push_back({p->d.plastic + (size_t)k * p->tet_cap, (size_t)tmax * 4});
            s.spans.push_back({p->d.plastic_c + (size_t)k * p->tet_cap, (size_t)tmax * 4});
        }
        s.spans.push_back({p->d.disp, (size_t)nmax * 16});
        s.spans.push_back({p->d.disp_c, (size_t)nmax * 16});
        s.spans.push_back({p->d.velocity, (size_t)nmax * 12});
        s.spans.push_back({p->d.meshes, (size_t)p->max_meshes * sizeof(PoolMesh)});
        s.spans.push_back({p->d.e_diss, (size_t)pmax * 8});
        s.spans.push_back({p->d.e_strain, (size_t)pmax * 8});
        s.spans.push_back({p->d.n_work, (size_t)pmax * 8});
        s.spans.push_back({p->d.n_kin, (size_t)pmax * 8});
        size_t total = 0;
        for (auto& sp : s.spans) total += sp.second;
        const int rc = check(p, fs::device_alloc((void**)&s.buf, total ? total : 1), "snapshot");
        if (rc) return rc;
    }
    size_t off = 0;
    for (auto& sp : s.spans) {
        if (restore)
            cudaMemcpyAsync(sp.first, s.buf + off, sp.second, cudaMemcpyDeviceToDevice, p->stream);
        else
            cudaMemcpyAsync(s.buf + off, sp.first, sp.second, cudaMemcpyDeviceToDevice, p->stream);
        off += sp.second;
    }
    return check(p, cudaStreamSynchronize(p->stream), "snapshot copy");
}

int wait_chunk(femstep_pool* p, double* gpu_ms) {
    if (gpu_ms) *gpu_ms = 0.0;
    if (!p->in_flight) return FEMSTEP_OK;
    p->in_flight = false;
    int rc = check(p, cudaEventSynchronize(p->ev1), "pool step");
    if (rc) return rc;
    if (*p->h_error) {
        // a grid barrier or a staged tile's copies gave up: the launch's outputs are
        // undefined, so the pool takes no further step
        p->broken = true;
        return fail(p, FEMSTEP_ETIMEOUT, "a device-side wait gave up (a grid barrier of the persistent launch, or a "
                                         "staged tile's copies); the pool's state is undefined and it takes no "
                                         "further step");
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, p->ev0, p->ev1);
    if (gpu_ms) *gpu_ms = ms;
    return FEMSTEP_OK;
}

int refresh_mirror(femstep_pool* p) {
    return check(p, cudaMemcpyAsync(p->h_meshes, p->d.meshes, sizeof(PoolMesh) * p->max_meshes,
                                    cudaMemcpyDeviceToHost, p->stream), "mesh table");
}

// ---- admission -------------------------------------------------------------------

// Where one admitted mesh goes, and where its staged arrays sit in the pinned buffer.
struct Placement {
    int id = -1;
    long long T = 0, N = 0, t0 = -1, n0 = -1, part0 = -1, e_tiles = 0, n_tiles = 0;
    size_t idx4 = 0, slot4 = 0, offs = 0, pos = 0, fixed = 0, ext = 0, rec = 0, end = 0;
    int status = FEMSTEP_OK;
    std::string what;
};

size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

// Offsets of a mesh's staged arrays, from `base`.
void stage_layout(Placement& pl, size_t base) {
    const size_t T = pl.T, N1 = pl.N + 1;
    size_t o = base;
    auto take = [&](size_t bytes) {
        const size_t at = o;
        o += align256(bytes);
        return at;
    };
    pl.idx4 = take(T * 16);
    pl.slot4 = take(T * 16);
    pl.offs = take(N1 * 4);
    pl.pos = take(N1 * 12);
    pl.fixed = take(N1);
    pl.ext = take(N1 * 12);
    pl.rec = take(sizeof(PoolMesh));
    pl.end = o;
}

// The host part of admitting one mesh, into its staged arrays (pinned): the CSR in the
// reference's order (fem.cpp:147-157), the slot map, the rest positions, pins and load;
// node and slot ids rebased into the pool.  The FP64 rest state (Dm^-1, volumes, lumped
// masses; fem.cpp:119-158) is computed on the device from the staged positions
// (launch_pool_admit).  Runs on any host thread; touches nothing but the mesh's
// own staging.
void prepare_mesh(const femstep_pool_mesh& m, Placement& pl, char* stage) {
    const long long N = pl.N, T = pl.T;
    std::vector<uint32_t> off, entry;
    fs::build_csr((size_t)N, (size_t)T, 4, m.index, off, entry);
    const long long s0 = 4 * pl.t0, n0 = pl.n0;
    uint4* idx4 = (uint4*)(stage + pl.idx4);
    uint4* slot4 = (uint4*)(stage + pl.slot4);
    {
        std::vector<uint32_t> sl(T * 4);
        for (long long n = 0; n < N; ++n)
            for (uint32_t k = off[n]; k < off[n + 1]; ++k) sl[entry[k]] = (uint32_t)(s0 + k);
        for (long long t = 0; t < T; ++t) {
            idx4[t] = make_uint4((uint32_t)(n0 + m.index[t * 4]), (uint32_t)(n0 + m.index[t * 4 + 1]),
                                 (uint32_t)(n0 + m.index[t * 4 + 2]), (uint32_t)(n0 + m.index[t * 4 + 3]));
            slot4[t] = make_uint4(sl[t * 4], sl[t * 4 + 1], sl[t * 4 + 2], sl[t * 4 + 3]);
        }
    }
    uint32_t* offs = (uint32_t*)(stage + pl.offs);
    for (long long n = 0; n <= N; ++n) offs[n] = (uint32_t)(s0 + off[n]);
    float* pos = (float*)(stage + pl.pos);
    std::memcpy(pos, m.position, (size_t)N * 12);
    uint8_t* fixed = (uint8_t*)(stage + pl.fixed);
    float* ext = (float*)(stage + pl.ext);
    for (long long n = 0; n < N; ++n) {
        fixed[n] = m.fixed && m.fixed[n] ? 1 : 0;
        for (int k = 0; k < 3; ++k) ext[n * 3 + k] = m.external_force ? (float)m.external_force[n * 3 + k] : 0.0f;
    }
    // the spare node slot: holds the CSR end; massless (set on the device), fixed, unloaded
    pos[N * 3] = pos[N * 3 + 1] = pos[N * 3 + 2] = 0.0f;
    fixed[N] = 1;
    ext[N * 3] = ext[N * 3 + 1] = ext[N * 3 + 2] = 0.0f;
}

// The host part of admitting one mesh of a group whose meshes sit in consecutive tet and
// node ranges (group_prepare / the device CSR): its node ids local to the group's node
// span, rest positions, pins and load, each into the group's section for it.  No CSR
// here: the device builds the group's (build_csr_device).
void prepare_mesh_sections(const femstep_pool_mesh& m, const Placement& pl, long long t_first, long long n_first,
                           char* idx_sec, char* pos_sec, char* fix_sec, char* ext_sec) {
    const long long N = pl.N, T = pl.T;
    const uint32_t shift = (uint32_t)(pl.n0 - n_first);
    uint32_t* idx = (uint32_t*)idx_sec + (pl.t0 - t_first) * 4;
    for (long long i = 0; i < T * 4; ++i) idx[i] = m.index[i] + shift;
    const long long at = pl.n0 - n_first;
    float* pos = (float*)pos_sec + at * 3;
    std::memcpy(pos, m.position, (size_t)N * 12);
    uint8_t* fixed = (uint8_t*)fix_sec + at;
    float* ext = (float*)ext_sec + at * 3;
    for (long long n = 0; n < N; ++n) fixed[n] = m.fixed && m.fixed[n] ? 1 : 0;
    if (m.external_force)
        for (long long i = 0; i < N * 3; ++i) ext[i] = (float)m.external_force[i];
    else
        std::memset(ext, 0, (size_t)N * 12);
    // the spare node slot: holds the CSR end; massless (set on the device), fixed, unloaded
    pos[N * 3] = pos[N * 3 + 1] = pos[N * 3 + 2] = 0.0f;
    fixed[N] = 1;
    ext[N * 3] = ext[N * 3 + 1] = ext[N * 3 + 2] = 0.0f;
}

// Whether some tet of the mesh has a non-zero volume (computeRestState's guard leaves
// a degenerate tet without stiffness; a mesh of them only has no time step).
bool any_volume(const femstep_pool_mesh& m) {
    for (size_t t = 0; t < m.tets; ++t) {
        const uint32_t* idx = &m.index[t * 4];
        double a[3][3];
        for (int c = 0; c < 3; ++c)
            for (int r = 0; r < 3; ++r)
                a[r][c] = (double)m.position[(size_t)idx[c + 1] * 3 + r] - (double)m.position[(size_t)idx[0] * 3 + r];
        const double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) -
                           a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
                           a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
        if (det != 0.0) return true;
    }
    return false;
}

// Run f(0..count-1) on the host's cores, largest work first (`weight`).
template <class F>
void parallel_for(int count, const std::vector<long long>& weight, F f) {
    std::vector<int> order(count);
    for (int i = 0; i < count; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return weight[a] > weight[b]; });
    const int workers = (int)std::min<unsigned>(std::max(1u, std::thread::hardware_concurrency()), (unsigned)count);
    if (workers <= 1) {
        for (int i : order) f(i);
        return;
    }
    std::atomic<int> next{0};
    std::vector<std::thread> pool;
    for (int w = 0; w < workers; ++w)
        pool.emplace_back([&]() {
            for (int k; (k = next.fetch_add(1)) < count;) f(order[k]);
        });
    for (auto& t : pool) t.join();
}

// Admit meshes[0..count) in order while they fit; *admitted = how many did.  Returns
// FEMSTEP_ENOMEM when some did not fit now, FEMSTEP_EINVAL (nothing admitted) when a
// mesh is not valid.
int admit_meshes(femstep_pool* p, const femstep_pool_mesh* meshes, const long long* steps, int count, int* ids,
                 int* admitted) {
    *admitted = 0;
    if (!p) return fail(p, FEMSTEP_EINVAL, "null pool");
    if (p->broken) return fail(p, FEMSTEP_ESTATE, "the pool stopped after a device wait gave up");
    for (int i = 0; i < count; ++i) {
        const femstep_pool_mesh& m = meshes[i];
        if (m.nodes == 0 || m.tets == 0 || !m.position || !m.index) return fail(p, FEMSTEP_EINVAL, "empty mesh");
        if (steps[i] < 0) return fail(p, FEMSTEP_EINVAL, "negative step count");
        if (!(m.density > 0.0)) return fail(p, FEMSTEP_EINVAL, "density must be positive");
        if (!(m.youngs_modulus > 0.0) || !(m.poisson_ratio > -1.0 && m.poisson_ratio < 0.5))
            return fail(p, FEMSTEP_EINVAL, "elastic constants out of range");
    }
    {
        // node ids in range, before anything is placed: an invalid mesh is invalid
        // whether or not it would fit
        std::vector<long long> weight(count);
        std::vector<char> bad(count, 0);
        for (int i = 0; i < count; ++i) weight[i] = (long long)meshes[i].tets;
        parallel_for(count, weight, [&](int i) {
            const femstep_pool_mesh& m = meshes[i];
            for (size_t k = 0; k < m.tets * 4; ++k)
                if (m.index[k] >= (uint32_t)m.nodes) {
                    bad[i] = 1;
                    return;
                }
            if (!any_volume(m)) bad[i] = 2;
        });
        for (int i = 0; i < count; ++i) {
            if (bad[i] == 1) return fail(p, FEMSTEP_EINVAL, "tet index out of range");
            if (bad[i] == 2) return fail(p, FEMSTEP_EINVAL, "every tet is degenerate");
        }
    }
    // places, in order, while they fit
    std::vector<Placement> pl;
    std::vector<bool> taken_id(p->max_meshes, false);
    int full = FEMSTEP_OK;
    std::string full_what;
    for (int i = 0; i < count; ++i) {
        const femstep_pool_mesh& m = meshes[i];
        Placement q;
        q.T = (long long)m.tets;
        q.N = (long long)m.nodes;
        q.e_tiles = (q.T + kMinTile - 1) / kMinTile;
        q.n_tiles = (q.N + kMinTile - 1) / kMinTile;
        for (int k = 0; k < p->max_meshes; ++k)
            if (!p->meshes[k].used && !taken_id[k]) {
                q.id = k;
                break;
            }
        if (q.id < 0) {
            full_what = "mesh table full";
        } else if ((q.t0 = p->tets.take(q.T)) < 0) {
            full_what = "no room for the tets now";
        } else if ((q.n0 = p->nodes.take(q.N + 1)) < 0) {
            p->tets.give(q.t0, q.T);
            full_what = "no room for the nodes now";
        } else if ((q.part0 = p->parts.take(q.e_tiles + q.n_tiles)) < 0) {
            p->tets.give(q.t0, q.T);
            p->nodes.give(q.n0, q.N + 1);
            full_what = "no room for the energy partials now";
        } else {
            taken_id[q.id] = true;
            pl.push_back(q);
            continue;
        }
        full = FEMSTEP_ENOMEM;
        break;
    }
    auto undo = [&]() {
        for (const Placement& q : pl) {
            p->tets.give(q.t0, q.T);
            p->nodes.give(q.n0, q.N + 1);
            p->parts.give(q.part0, q.e_tiles + q.n_tiles);
        }
    };
    const int n = (int)pl.size();
    if (n == 0) return full ? fail(p, full, full_what) : FEMSTEP_OK;
    // Groups of at most kStageGroup staged bytes (a larger mesh is a group alone): each
    // group is prepared on all cores into a pinned buffer and its copies queued, so a
    // group's host work overlaps the uploads of the one before, and the pinned memory
    // stays bounded (buffers are reused once their copies are done).
    constexpr size_t kStageGroup = size_t(64) << 20;
    PoolDevice& d = p->d;
    cudaStream_t st = p->stream;
    for (int g0 = 0; g0 < n;) {
        int g1 = g0;
        size_t bytes = 0;
        while (g1 < n) {
            stage_layout(pl[g1], bytes);
            if (g1 > g0 && pl[g1].end > kStageGroup) break;
            bytes = pl[g1].end;
            ++g1;
        }
        std::vector<long long> weight(g1 - g0);
        for (int i = g0; i < g1; ++i) weight[i - g0] = pl[i].T;
        const int G = g1 - g0;
        // A group in consecutive tet and node ranges, in order (always so in a pool that
        // was empty): staged by section and uploaded in one copy per section, its CSR
        // and slot map built on the device over the whole group -- the per-mesh
        // counting sorts, since every corner of a mesh names only that mesh's nodes.
        // Otherwise each mesh is prepared on the host and sent by its own copies.
        bool contig = true;
        for (int i = g0 + 1; i < g1; ++i)
            contig = contig && pl[i].t0 == pl[i - 1].t0 + pl[i - 1].T && pl[i].n0 == pl[i - 1].n0 + pl[i - 1].N + 1;
        long long tets_g = 0, nodes_g = 0;
        for (int i = g0; i < g1; ++i) {
            tets_g += pl[i].T;
            nodes_g += pl[i].N + 1;
        }
        size_t sec_idx = 0, sec_pos = 0, sec_fix = 0, sec_ext = 0, sec_rec = 0;
        if (contig) {
            size_t o = 0;
            sec_idx = o, o += align256((size_t)tets_g * 16);
            sec_pos = o, o += align256((size_t)nodes_g * 12);
            sec_fix = o, o += align256((size_t)nodes_g);
            sec_ext = o, o += align256((size_t)nodes_g * 12);
            sec_rec = o, o += align256((size_t)G * sizeof(PoolMesh));
            bytes = o;
        }
        const size_t table = ((size_t)G * sizeof(fs::PoolAdmit) + 255) & ~size_t(255);
        cudaError_t err;
        Staging::Buf* buf = p->staging.get(bytes + table, err);
        if (!buf) {
            undo();  // earlier groups' copies went to ranges that are free again
            return check(p, err, "pinned staging");
        }
        char* stage = Staging::take(buf, bytes);
        fs::PoolAdmit* adm = (fs::PoolAdmit*)Staging::take(buf, table);
        const long long t_first = pl[g0].t0, n_first = pl[g0].n0;
        if (contig) {
            parallel_for(g1 - g0, weight, [&](int k) {
                prepare_mesh_sections(meshes[g0 + k], pl[g0 + k], t_first, n_first, stage + sec_idx, stage + sec_pos,
                                      stage + sec_fix, stage + sec_ext);
                // the host copy of the rest positions, for the readback
                p->meshes[pl[g0 + k].id].rest.assign(meshes[g0 + k].position,
                                                     meshes[g0 + k].position + pl[g0 + k].N * 3);
            });
        } else {
            parallel_for(g1 - g0, weight, [&](int k) {
                prepare_mesh(meshes[g0 + k], pl[g0 + k], stage);
                p->meshes[pl[g0 + k].id].rest.assign(meshes[g0 + k].position,
                                                     meshes[g0 + k].position + pl[g0 + k].N * 3);
            });
        }
        long long tets = 0, nodes = 0, parts = 0;
        bool any_dt = false;
        auto send = [&](void* dst, size_t off, size_t len) {
            cudaMemcpyAsync(dst, stage + off, len, cudaMemcpyHostToDevice, st);
        };
        if (contig) {
            send(d.index + t_first, sec_idx, (size_t)tets_g * 16);
            send(d.velocity + n_first * 3, sec_pos, (size_t)nodes_g * 12);
            send(d.fixed + n_first, sec_fix, (size_t)nodes_g);
            send(d.ext + n_first * 3, sec_ext, (size_t)nodes_g * 12);
            // the group's last node is its last mesh's spare slot, which holds the CSR end
            const cudaError_t ce = fs::build_csr_device(reinterpret_cast<const uint32_t*>(d.index + t_first),
                                                        tets_g * 4, nodes_g - 1, d.offset + n_first,
                                                        reinterpret_cast<uint32_t*>(d.slot + t_first), st, nullptr,
                                                        (uint32_t)(4 * t_first));
            if (ce != cudaSuccess) {
                undo();
                return check(p, ce, "group adjacency");
            }
            fs::launch_pool_rebase(d.index + t_first, tets_g, (uint32_t)n_first, st);
        }
        for (int i = g0; i < g1; ++i) {
            const femstep_pool_mesh& m = meshes[i];
            const Placement& q = pl[i];
            const long long T = q.T, N = q.N, t0 = q.t0, n0 = q.n0, part0 = q.part0;
            if (!contig) {
                send(d.index + t0, q.idx4, T * sizeof(uint4));
                send(d.slot + t0, q.slot4, T * sizeof(uint4));
                send(d.offset + n0, q.offs, (N + 1) * 4);
                send(d.fixed + n0, q.fixed, N + 1);
                send(d.ext + n0 * 3, q.ext, (N + 1) * 12);
                // the rest positions, staged in the mesh's velocity rows for the rest
                // state; the admission kernels below then start the nodes at rest
                send(d.velocity + n0 * 3, q.pos, (N + 1) * 12);
            }
            const size_t rec_at = contig ? sec_rec + (size_t)(i - g0) * sizeof(PoolMesh) : q.rec;
            PoolMesh* pm = (PoolMesh*)(stage + rec_at);
            std::memset(pm, 0, sizeof(PoolMesh));
            const double E = m.youngs_modulus, nu = m.poisson_ratio;
            // plasticity::Material::shearModulus / bulkModulus (plasticity.hpp:226-227)
            pm->mat = fs::make_j2f(E / (2.0 * (1.0 + nu)), E / (3.0 * (1.0 - 2.0 * nu)), m.yield_strength,
                                   m.hardening_modulus);
            pm->dt64 = m.dt > 0.0 ? m.dt : 0.0;
            pm->dt = (float)pm->dt64;
            pm->gravity = (float)m.gravity;
            pm->damping = (float)(m.damping > 0.0 ? m.damping : 1.0);
            pm->ramp = m.ramp_steps;
            pm->step = 0;
            pm->target = steps[i];
            pm->e_part = part0;
            pm->n_part = part0 + q.e_tiles;
            pm->serial = p->next_serial + i;
            send(d.meshes + q.id, rec_at, sizeof(PoolMesh));
            // the group's record of this mesh for the admission kernels; no step given:
            // 0.9 x the FP64 element eigenvalue bound of the stored FP32 Dm^-1, formed
            // and stored on the device behind the uploads
            fs::PoolAdmit& a = adm[i - g0];
            a.t0 = t0;
            a.T = T;
            a.n0 = n0;
            a.N = N;
            a.part0 = part0;
            a.parts = q.e_tiles + q.n_tiles;
            a.tet_first = tets;
            a.node_first = nodes;
            a.part_first = parts;
            a.density = m.density;
            a.lambda = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
            a.mu = E / (2.0 * (1.0 + nu));
            a.id = q.id;
            a.want_dt = m.dt > 0.0 ? 0 : 1;
            any_dt = any_dt || a.want_dt;
            tets += T;
            nodes += N + 1;
            parts += a.parts;
        }
        cudaMemcpyAsync(p->d_admit, adm, (size_t)G * sizeof(fs::PoolAdmit), cudaMemcpyHostToDevice, st);
        fs::launch_pool_admit(d, p->d_admit, G, tets, nodes, parts, any_dt, p->d_w2, st);
        Staging::submit(buf, st);
        g0 = g1;
    }
    const int rc = check(p, cudaGetLastError(), "admit upload");
    if (rc) {
        undo();
        return rc;
    }
    for (int i = 0; i < n; ++i) {
        const Placement& q = pl[i];
        HostMesh& h = p->meshes[q.id];
        h.used = true;
        h.t0 = q.t0;
        h.T = q.T;
        h.n0 = q.n0;
        h.N = q.N;
        h.e_part = q.part0;
        h.n_part = q.part0 + q.e_tiles;
        h.e_tiles = q.e_tiles;
        h.n_tiles = q.n_tiles;
        h.target = steps[i];
        h.serial = p->next_serial + i;
        ids[i] = q.id;
    }
    p->next_serial += n;
    p->dirty = true;
    *admitted = n;
    return full ? fail(p, full, full_what) : FEMSTEP_OK;
}

}  // namespace

extern "C" {

int femstep_pool_create(size_t tet_capacity, size_t node_capacity, int max_meshes, int tile, femstep_pool** out) {
    if (out) *out = nullptr;
    if (!out || tet_capacity == 0 || node_capacity == 0 || max_meshes <= 0)
        return fail(nullptr, FEMSTEP_EINVAL, "empty pool");
    if (tet_capacity > 1000000000ull) return fail(nullptr, FEMSTEP_EINVAL, "tet capacity above 1e9 (32-bit slot ids)");
    if (node_capacity > 2000000000ull) return fail(nullptr, FEMSTEP_EINVAL, "node capacity above 2e9");
    if (tile == 0) tile = 256;
    if (tile != 128 && tile != 256 && tile != 512) return fail(nullptr, FEMSTEP_EINVAL, "tile must be 128, 256 or 512");
    const int dev = fs::device_status();
    if (dev != FEMSTEP_OK) return dev;
    fs::pool_kernels_setup();
    femstep_pool* p = new femstep_pool();
    // rows of 4-byte per-tet data start on 16-byte boundaries (bulk copies need them)
    tet_capacity = (tet_capacity + 3) & ~size_t(3);
    p->tet_cap = (long long)tet_capacity;
    p->node_cap = (long long)node_capacity;
    p->max_meshes = max_meshes;
    p->tile = tile;
    // partial slots: every mesh reserves ceil(T/128) + ceil(N/128) (the smallest tile)
    p->part_cap = (long long)(tet_capacity + node_capacity) / kMinTile + 2LL * max_meshes;
    int rc = check(p, cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking), "stream");
    if (!rc) rc = check(p, cudaEventCreate(&p->ev0), "event");
    if (!rc) rc = check(p, cudaEventCreate(&p->ev1), "event");
    if (!rc) rc = check(p, cudaHostAlloc(&p->h_meshes, sizeof(PoolMesh) * max_meshes, cudaHostAllocDefault), "pinned");
    if (!rc) rc = check(p, cudaHostAlloc(&p->h_error, sizeof(int), cudaHostAllocDefault), "pinned");
    if (rc) {
        femstep_pool_destroy(p);
        return rc;
    }
    std::memset(p->h_meshes, 0, sizeof(PoolMesh) * max_meshes);
    *p->h_error = 0;
    fs::DeviceArena& A = p->arena;
    PoolDevice& d = p->d;
    const size_t Tc = tet_capacity, Nc = node_capacity;
    d.tet_cap = (long long)Tc;
    d.node_cap = (long long)Nc;
    d.index = A.zeros<uint4>(Tc);
    d.slot = A.zeros<uint4>(Tc);
    d.rest_inv = A.alloc<float>(Tc * 9);
    d.rest_vol = A.alloc<float>(Tc);
    d.plastic = A.alloc<float>(Tc * 7);
    d.plastic_c = A.alloc<float>(Tc * 7);
    d.slots = A.alloc<float4>(Tc * 4 + 1);
    d.offset = A.zeros<uint32_t>(Nc);
    d.disp = A.alloc<float4>(Nc);
    d.disp_c = A.alloc<float4>(Nc);
    d.velocity = A.alloc<float>(Nc * 3);
    d.mass = A.alloc<float>(Nc);
    d.inv_mass = A.alloc<float>(Nc);
    d.fixed = A.zeros<uint8_t>(Nc);
    d.ext = A.zeros<float>(Nc * 3);
    d.meshes = A.zeros<PoolMesh>(max_meshes);
    d.e_diss = A.zeros<double>(p->part_cap);
    d.e_strain = A.zeros<double>(p->part_cap);
    d.n_work = A.zeros<double>(p->part_cap);
    d.n_kin = A.zeros<double>(p->part_cap);
    d.barrier = A.zeros<unsigned int>(2);
    d.error = A.zeros<int>(1);
    p->d_etiles = A.alloc<PoolTile>(p->part_cap);
    p->d_ntiles = A.alloc<PoolTile>(p->part_cap);
    p->d_active = A.zeros<int>(max_meshes);
    p->d_admit = A.alloc<fs::PoolAdmit>(max_meshes);
    p->d_w2 = A.zeros<unsigned long long>(max_meshes);
    p->d_out = A.zeros<double>(8);
    if (!A.ok()) {
        const int code = A.status() == cudaErrorMemoryAllocation ? FEMSTEP_ENOMEM : FEMSTEP_ECUDA;
        fail(p, code, std::string("pool allocation failed: ") + cudaGetErrorString(A.status()));
        femstep_pool_destroy(p);
        return code;
    }
    p->tets.reset(p->tet_cap);
    p->nodes.reset(p->node_cap);
    p->parts.reset(p->part_cap);
    p->meshes.resize(max_meshes);
    *out = p;
    return FEMSTEP_OK;
}

size_t femstep_pool_bytes_per_tet(void) { return 16 + 16 + 36 + 4 + 28 + 28 + 64; }
size_t femstep_pool_bytes_per_node(void) { return 4 + 16 + 16 + 12 + 4 + 4 + 1 + 12; }

int femstep_pool_admit(femstep_pool* p, const femstep_pool_mesh* mesh, long long steps, int* id) {
    if (!id) return fail(p, FEMSTEP_EINVAL, "null argument");
    int admitted = 0;
    return admit_meshes(p, mesh, &steps, 1, id, &admitted);
}

int femstep_pool_admit_many(femstep_pool* p, const femstep_pool_mesh* meshes, const long long* steps, int count,
                            int* ids, int* admitted) {
    if (admitted) *admitted = 0;
    if (!admitted || (count > 0 && (!meshes || !steps || !ids))) return fail(p, FEMSTEP_EINVAL, "null argument");
    return admit_meshes(p, meshes, steps, count, ids, admitted);
}

int femstep_pool_release(femstep_pool* p, int id) {
    if (!valid_id(p, id)) return fail(p, FEMSTEP_EINVAL, "unknown mesh");
    HostMesh& h = p->meshes[id];
    // freeze it behind any queued work, so no work list can touch the ranges again
    cudaMemsetAsync(p->d.meshes + id, 0, sizeof(PoolMesh), p->stream);
    p->tets.give(h.t0, h.T);
    p->nodes.give(h.n0, h.N + 1);
    p->parts.give(h.e_part, h.e_tiles + h.n_tiles);
    h = HostMesh{};
    p->dirty = true;
    return check(p, cudaGetLastError(), "release");
}

// ---- eviction: checkpoint one mesh, bring it back later ----
//
// A mesh's mutable state in the pool -- displacement and its compensation, velocity,
// plastic strain and its compensation, its energy partial slots and its record (step
// counter, step size) -- as one host buffer.  admit_resume admits the same mesh again
// (anywhere in the pool) and puts the state back; it then steps on exactly as if it
// had never left, since no per-tet or per-node arithmetic depends on where a mesh
// sits or who its neighbours are.

namespace {

constexpr uint64_t kPoolCheckpointMagic = 0x3150484c4f4f5046ull;  // "FPOOLHP1"

struct PoolCheckpointHeader {
    uint64_t magic;
    int64_t T, N, e_tiles, n_tiles, tile;
    PoolMesh rec;
};

struct PoolSegment {
    void* dev;      // device address
    size_t bytes;
};

std::vector<PoolSegment> pool_segments(femstep_pool* p, const HostMesh& h) {
    PoolDevice& d = p->d;
    std::vector<PoolSegment> v = {
        {d.disp + h.n0, (size_t)(h.N + 1) * sizeof(float4)},
        {d.disp_c + h.n0, (size_t)(h.N + 1) * sizeof(float4)},
        {d.velocity + h.n0 * 3, (size_t)(h.N + 1) * 3 * sizeof(float)},
    };
    for (int k = 0; k < 7; ++k) v.push_back({d.plastic + (size_t)k * p->tet_cap + h.t0, (size_t)h.T * sizeof(float)});
    for (int k = 0; k < 7; ++k) v.push_back({d.plastic_c + (size_t)k * p->tet_cap + h.t0, (size_t)h.T * sizeof(float)});
    v.push_back({d.e_diss + h.e_part, (size_t)h.e_tiles * sizeof(double)});
    v.push_back({d.e_strain + h.e_part, (size_t)h.e_tiles * sizeof(double)});
    v.push_back({d.n_work + h.n_part, (size_t)h.n_tiles * sizeof(double)});
    v.push_back({d.n_kin + h.n_part, (size_t)h.n_tiles * sizeof(double)});
    return v;
}

size_t pool_checkpoint_bytes(femstep_pool* p, const HostMesh& h) {
    size_t total = sizeof(PoolCheckpointHeader);
    for (const PoolSegment& g : pool_segments(p, h)) total += g.bytes;
    return total;
}

}  // namespace

int femstep_pool_checkpoint_size(femstep_pool* p, int id, size_t* bytes) {
    if (!valid_id(p, id) || !bytes) return fail(p, FEMSTEP_EINVAL, "unknown mesh");
    *bytes = pool_checkpoint_bytes(p, p->meshes[id]);
    return FEMSTEP_OK;
}

int femstep_pool_checkpoint(femstep_pool* p, int id, void* buffer, size_t bytes) {
    if (!valid_id(p, id) || !buffer) return fail(p, FEMSTEP_EINVAL, "unknown mesh");
    if (p->in_flight) return fail(p, FEMSTEP_ESTATE, "a chunk is running: wait for it first");
    const HostMesh& h = p->meshes[id];
    if (bytes < pool_checkpoint_bytes(p, h)) return fail(p, FEMSTEP_EINVAL, "checkpoint buffer too small");
    PoolCheckpointHeader hd{};
    hd.magic = kPoolCheckpointMagic;
    hd.T = h.T;
    hd.N = h.N;
    hd.e_tiles = h.e_tiles;
    hd.n_tiles = h.n_tiles;
    hd.tile = p->tile;
    int rc = check(p, cudaMemcpyAsync(&hd.rec, p->d.meshes + id, sizeof(PoolMesh), cudaMemcpyDeviceToHost, p->stream),
                   "checkpoint");
    char* out = static_cast<char*>(buffer) + sizeof(hd);
    for (const PoolSegment& g : pool_segments(p, h)) {
        if (!rc) rc = check(p, cudaMemcpyAsync(out, g.dev, g.bytes, cudaMemcpyDeviceToHost, p->stream), "checkpoint");
        out += g.bytes;
    }
    if (!rc) rc = check(p, cudaStreamSynchronize(p->stream), "checkpoint");
    if (rc) return rc;
    std::memcpy(buffer, &hd, sizeof(hd));
    return FEMSTEP_OK;
}

int femstep_pool_admit_resume(femstep_pool* p, const femstep_pool_mesh* mesh, long long steps, const void* buffer,
                              size_t bytes, int* id) {
    if (!p || !mesh || !buffer || !id) return fail(p, FEMSTEP_EINVAL, "null argument");
    PoolCheckpointHeader hd;
    if (bytes < sizeof(hd)) return fail(p, FEMSTEP_EINVAL, "not a pool checkpoint");
    std::memcpy(&hd, buffer, sizeof(hd));
    if (hd.magic != kPoolCheckpointMagic) return fail(p, FEMSTEP_EINVAL, "not a pool checkpoint");
    if (hd.T != (int64_t)mesh->tets || hd.N != (int64_t)mesh->nodes)
        return fail(p, FEMSTEP_EINVAL, "checkpoint of a different mesh");
    if (steps < hd.rec.step) return fail(p, FEMSTEP_EINVAL, "target below the steps already taken");
    int admitted = 0;
    int rc = admit_meshes(p, mesh, &steps, 1, id, &admitted);
    if (rc || admitted != 1) return rc ? rc : fail(p, FEMSTEP_ENOMEM, "no room now");
    HostMesh& h = p->meshes[*id];
    if (bytes < pool_checkpoint_bytes(p, h) || hd.e_tiles != h.e_tiles || hd.n_tiles != h.n_tiles) {
        femstep_pool_release(p, *id);
        return fail(p, FEMSTEP_EINVAL, "checkpoint size does not match this mesh");
    }
    // behind the admission's own uploads on the stream: the state, then the record with
    // this placement's partial slots, serial and target
    const char* in = static_cast<const char*>(buffer) + sizeof(hd);
    for (const PoolSegment& g : pool_segments(p, h)) {
        if (!rc) rc = check(p, cudaMemcpyAsync(g.dev, in, g.bytes, cudaMemcpyHostToDevice, p->stream), "resume");
        in += g.bytes;
    }
    PoolMesh rec = hd.rec;
    rec.e_part = h.e_part;
    rec.n_part = h.n_part;
    rec.serial = h.serial;
    rec.target = steps;
    if (!rc) rc = check(p, cudaMemcpyAsync(p->d.meshes + *id, &rec, sizeof(rec), cudaMemcpyHostToDevice, p->stream),
                        "resume");
    if (!rc) rc = check(p, cudaStreamSynchronize(p->stream), "resume");
    if (rc) {
        femstep_pool_release(p, *id);
        return rc;
    }
    return FEMSTEP_OK;
}

int femstep_pool_run_async(femstep_pool* p, int steps, int mode) {
    if (!p) return fail(p, FEMSTEP_EINVAL, "null pool");
    if (p->broken) return fail(p, FEMSTEP_ESTATE, "the pool stopped after a device wait gave up");
    if (steps < 0) return fail(p, FEMSTEP_EINVAL, "negative step count");
    if (p->in_flight) return fail(p, FEMSTEP_ESTATE, "a chunk is already running: wait for it first");
    if (mode == FEMSTEP_POOL_AUTO) mode = p->mode;
    if (!valid_mode(mode)) return fail(p, FEMSTEP_EINVAL, "bad mode");
    if (mode == FEMSTEP_POOL_GRAPH_TILED && p->tile != 128)
        return fail(p, FEMSTEP_EINVAL, "the tiled schedule runs tiles of 128");
    int rc = rebuild(p);
    if (rc) return rc;
    p->launches = 0;
    rc = check(p, cudaEventRecord(p->ev0, p->stream), "event");
    if (!rc) rc = launch_chunk(p, steps, mode);
    if (!rc) rc = refresh_mirror(p);
    if (!rc) rc = check(p, cudaMemcpyAsync(p->h_error, p->d.error, sizeof(int), cudaMemcpyDeviceToHost, p->stream),
                        "error flag");
    if (!rc) rc = check(p, cudaEventRecord(p->ev1, p->stream), "event");
    if (rc) return rc;
    p->in_flight = true;
    return FEMSTEP_OK;
}

int femstep_pool_prepare(femstep_pool* p) {
    if (!p) return fail(p, FEMSTEP_EINVAL, "null pool");
    if (p->broken) return fail(p, FEMSTEP_ESTATE, "the pool stopped after a device wait gave up");
    if (p->in_flight) return fail(p, FEMSTEP_ESTATE, "a chunk is running: wait for it first");
    int rc = rebuild(p);
    if (rc) return rc;
    if (p->d.n_etiles > 0 && p->mode != FEMSTEP_POOL_PERSISTENT)
        rc = ensure_graph(p, passes_of(p->mode));
    if (!rc) rc = check(p, cudaStreamSynchronize(p->stream), "prepare");
    return rc;
}

int femstep_pool_wait(femstep_pool* p, double* gpu_ms) {
    if (!p) return fail(p, FEMSTEP_EINVAL, "null pool");
    return wait_chunk(p, gpu_ms);
}

int femstep_pool_run(femstep_pool* p, int steps, int mode, double* gpu_ms) {
    const int rc = femstep_pool_run_async(p, steps, mode);
    if (rc) return rc;
    return wait_chunk(p, gpu_ms);
}

int femstep_pool_finished(femstep_pool* p, int* ids, int capacity, int* count) {
    if (!p || !count || (capacity > 0 && !ids)) return fail(p, FEMSTEP_EINVAL, "null argument");
    if (p->in_flight) return fail(p, FEMSTEP_ESTATE, "a chunk is running: wait for it first");
    int n = 0;
    for (int id = 0; id < p->max_meshes; ++id) {
        const HostMesh& h = p->meshes[id];
        if (!h.used) continue;
        // the mirror is as of the last chunk: a record of an earlier tenant of this id,
        // or none yet, carries another serial
        const PoolMesh& r = p->h_meshes[id];
        if (r.serial == h.serial && r.step >= r.target) {
            if (n < capacity) ids[n] = id;
            ++n;
        }
    }
    *count = n;
    return FEMSTEP_OK;
}

int femstep_pool_status(femstep_pool* p, int id, long long* steps_done, long long* steps_target) {
    if (!valid_id(p, id)) return fail(p, FEMSTEP_EINVAL, "unknown mesh");
    std::vector<PoolMesh> r(1);
    int rc = check(p, cudaMemcpyAsync(r.data(), p->d.meshes + id, sizeof(PoolMesh), cudaMemcpyDeviceToHost,
                                      p->stream), "status");
    if (!rc) rc = check(p, cudaStreamSynchronize(p->stream), "status");
    if (!rc) {
        if (steps_done) *steps_done = r[0].step;
        if (steps_target) *steps_target = r[0].target;
    }
    return rc;
}

int femstep_pool_readback(femstep_pool* p, int id, double* position, double* velocity) {
    if (!valid_id(p, id)) return fail(p, FEMSTEP_EINVAL, "unknown mesh");
    const HostMesh& h = p->meshes[id];
    std::vector<float4> u(h.N), c(h.N);
    std::vector<float> v(h.N * 3);
    int rc = check(p, cudaMemcpyAsync(u.data(), p->d.disp + h.n0, h.N * 16, cudaMemcpyDeviceToHost, p->stream),
                   "readback");
    if (!rc)
        rc = check(p, cudaMemcpyAsync(c.data(), p->d.disp_c + h.n0, h.N * 16, cudaMemcpyDeviceToHost, p->stream),
                   "readback");
    if (!rc)
        rc = check(p, cudaMemcpyAsync(v.data(), p->d.velocity + h.n0 * 3, v.size() * 4, cudaMemcpyDeviceToHost,
                                      p->stream), "readback");
    if (!rc) rc = check(p, cudaStreamSynchronize(p->stream), "readback");
    if (rc) return rc;
    // the compensated displacement u - c, in double
    if (position)
        for (long long n = 0; n < h.N; ++n) {
            position[n * 3] = (double)h.rest[n * 3] + ((double)u[n].x - (double)c[n].x);
            position[n * 3 + 1] = (double)h.rest[n * 3 + 1] + ((double)u[n].y - (double)c[n].y);
            position[n * 3 + 2] = (double)h.rest[n * 3 + 2] + ((double)u[n].z - (double)c[n].z);
        }
    if (velocity)
        for (size_t i = 0; i < v.size(); ++i) velocity[i] = v[i];
    return FEMSTEP_OK;
}

int femstep_pool_readback_many(femstep_pool* p, int count, const int* ids, double* const* positions,
                               double* const* velocities) {
    if (!p || count < 0 || (count > 0 && (!ids || !positions))) return fail(p, FEMSTEP_EINVAL, "null argument");
    for (int i = 0; i < count; ++i)
        if (!valid_id(p, ids[i])) return fail(p, FEMSTEP_EINVAL, "unknown mesh");
    // Groups of at most 64 MB: each group's node rows go device -> pinned staging in three
    // copies per mesh, all groups queued at once; then each group is converted on all host
    // cores as soon as its copies have landed, while the later groups are still copying.
    constexpr size_t kGroup = size_t(64) << 20;
    struct Group {
        int first = 0, last = 0;
        Staging::Buf* buf = nullptr;
        std::vector<size_t> at;  // per mesh: offset of its rows in the buffer
    };
    std::vector<Group> groups;
    for (int i = 0; i < count;) {
        Group g;
        g.first = i;
        size_t bytes = 0;
        while (i < count) {
            const size_t b = (size_t)p->meshes[ids[i]].N * 44 + 3 * 256;
            if (i > g.first && bytes + b > kGroup) break;
            bytes += b;
            ++i;
        }
        g.last = i;
        cudaError_t err;
        g.buf = p->staging.get(bytes, err);
        if (!g.buf) return check(p, err, "pinned staging");
        for (int k = g.first; k < g.last; ++k) {
            const HostMesh& h = p->meshes[ids[k]];
            char* u = Staging::take(g.buf, (size_t)h.N * 16);
            char* c = Staging::take(g.buf, (size_t)h.N * 16);
            char* v = Staging::take(g.buf, (size_t)h.N * 12);
            g.at.push_back((size_t)(u - g.buf->host));
            cudaMemcpyAsync(u, p->d.disp + h.n0, h.N * 16, cudaMemcpyDeviceToHost, p->stream);
            cudaMemcpyAsync(c, p->d.disp_c + h.n0, h.N * 16, cudaMemcpyDeviceToHost, p->stream);
            cudaMemcpyAsync(v, p->d.velocity + h.n0 * 3, h.N * 12, cudaMemcpyDeviceToHost, p->stream);
        }
        Staging::submit(g.buf, p->stream);
        groups.push_back(std::move(g));
    }
    int rc = check(p, cudaGetLastError(), "readback");
    if (rc) return rc;
    for (Group& g : groups) {
        rc = check(p, cudaEventSynchronize(g.buf->done), "readback");
        if (rc) return rc;
        const int n = g.last - g.first;
        std::vector<long long> weight(n);
        for (int k = 0; k < n; ++k) weight[k] = p->meshes[ids[g.first + k]].N;
        parallel_for(n, weight, [&](int k) {
            const HostMesh& h = p->meshes[ids[g.first + k]];
            const char* base = g.buf->host + g.at[k];
            const float4* u = reinterpret_cast<const float4*>(base);
            const float4* c = reinterpret_cast<const float4*>(base + ((h.N * 16 + 255) & ~255LL));
            const float* v = reinterpret_cast<const float*>(base + 2 * ((h.N * 16 + 255) & ~255LL));
            double* pos = positions[g.first + k];
            double* vel = velocities ? velocities[g.first + k] : nullptr;
            for (long long i = 0; i < h.N; ++i) {
                // the compensated displacement u - c, in double
                pos[i * 3] = (double)h.rest[i * 3] + ((double)u[i].x - (double)c[i].x);
                pos[i * 3 + 1] = (double)h.rest[i * 3 + 1] + ((double)u[i].y - (double)c[i].y);
                pos[i * 3 + 2] = (double)h.rest[i * 3 + 2] + ((double)u[i].z - (double)c[i].z);
            }
            if (vel)
                for (long long i = 0; i < h.N * 3; ++i) vel[i] = v[i];
        });
    }
    return FEMSTEP_OK;
}

int femstep_pool_plastic(femstep_pool* p, int id, double* plastic) {
    if (!valid_id(p, id) || !plastic) return fail(p, FEMSTEP_EINVAL, "unknown mesh");
    const HostMesh& h = p->meshes[id];
    std::vector<float> buf((size_t)h.T * 7);
    int rc = FEMSTEP_OK;
    for (int k = 0; k < 7 && !rc; ++k)
        rc = check(p, cudaMemcpyAsync(buf.data() + (size_t)k * h.T, p->d.plastic + (size_t)k * p->tet_cap + h.t0,
                                      h.T * 4, cudaMemcpyDeviceToHost, p->stream), "readback");
    if (!rc) rc = check(p, cudaStreamSynchronize(p->stream), "readback");
    if (rc) return rc;
    for (long long t = 0; t < h.T; ++t)
        for (int k = 0; k < 7; ++k) plastic[t * 7 + k] = buf[(size_t)k * h.T + t];
    return FEMSTEP_OK;
}

int femstep_pool_energy(femstep_pool* p, int id, double out[4]) {
    if (!valid_id(p, id) || !out) return fail(p, FEMSTEP_EINVAL, "unknown mesh");
    const HostMesh& h = p->meshes[id];
    // accumulated terms: every slot the mesh holds (a slot no tiling touched is 0);
    // instantaneous terms: the slots of the current tiling
    const long long et = (h.T + p->tile - 1) / p->tile, nt = (h.N + p->tile - 1) / p->tile;
    fs::launch_reduce_sum(p->d.n_work + h.n_part, h.n_tiles, p->d_out + 0, p->stream);
    fs::launch_reduce_sum(p->d.e_diss + h.e_part, h.e_tiles, p->d_out + 1, p->stream);
    fs::launch_reduce_sum(p->d.e_strain + h.e_part, et, p->d_out + 2, p->stream);
    fs::launch_reduce_sum(p->d.n_kin + h.n_part, nt, p->d_out + 3, p->stream);
    std::vector<double> tmp(4);
    int rc = check(p, cudaGetLastError(), "reduce");
    if (!rc) rc = check(p, cudaMemcpyAsync(tmp.data(), p->d_out, 32, cudaMemcpyDeviceToHost, p->stream), "readback");
    if (!rc) rc = check(p, cudaStreamSynchronize(p->stream), "reduce");
    if (!rc) std::memcpy(out, tmp.data(), 32);
    return rc;
}

int femstep_pool_dt(femstep_pool* p, int id, double* dt) {
    if (!valid_id(p, id) || !dt) return fail(p, FEMSTEP_EINVAL, "unknown mesh");
    std::vector<PoolMesh> r(1);
    int rc = check(p, cudaMemcpyAsync(r.data(), p->d.meshes + id, sizeof(PoolMesh), cudaMemcpyDeviceToHost, p->stream),
                   "dt");
    if (!rc) rc = check(p, cudaStreamSynchronize(p->stream), "dt");
    if (!rc) *dt = r[0].dt64;
    return rc;
}

int femstep_pool_autotune(femstep_pool* p, int steps, int* tile_out, int* mode_out, double* ms_out) {
    if (!p || steps <= 0) return fail(p, FEMSTEP_EINVAL, "bad argument");
    if (p->broken) return fail(p, FEMSTEP_ESTATE, "the pool stopped after a device wait gave up");
    if (p->in_flight) return fail(p, FEMSTEP_ESTATE, "a chunk is running: wait for it first");
    Snapshot snap;
    int rc = snapshot(p, snap, false);
    if (rc) return rc;
    const int tiles[3] = {128, 256, 512};
    const int modes[4] = {FEMSTEP_POOL_GRAPH, FEMSTEP_POOL_PERSISTENT, FEMSTEP_POOL_GRAPH_STAGED,
                          FEMSTEP_POOL_GRAPH_TILED};
    const int tile0 = p->tile, mode0 = p->mode;
    double best = INFINITY;
    int best_tile = tile0, best_mode = mode0;
    for (int ti = 0; ti < 3 && !rc; ++ti)
        for (int mi = 0; mi < 4 && !rc; ++mi) {
            if (modes[mi] == FEMSTEP_POOL_GRAPH_STAGED && tiles[ti] == 512) continue;  // staged: 128, 256
            if (modes[mi] == FEMSTEP_POOL_GRAPH_TILED && tiles[ti] != 128) continue;   // tiled: 128
            p->tile = tiles[ti];
            p->dirty = true;
            double ms = 0.0;
            rc = femstep_pool_run(p, steps, modes[mi], &ms);  // warm (graph build, caches)
            if (!rc) rc = snapshot(p, snap, true);
            if (!rc) rc = femstep_pool_run(p, steps, modes[mi], &ms);
            if (!rc) rc = snapshot(p, snap, true);
            if (!rc && ms < best) {
                best = ms;
                best_tile = tiles[ti];
                best_mode = modes[mi];
            }
        }
    fs::device_free(snap.buf);
    p->tile = best_tile;
    p->mode = best_mode;
    p->dirty = true;
    if (rc) return rc;
    // the instantaneous partials of the other tilings are stale: zero them
    cudaMemsetAsync(p->d.e_strain, 0, (size_t)p->part_cap * 8, p->stream);
    cudaMemsetAsync(p->d.n_kin, 0, (size_t)p->part_cap * 8, p->stream);
    // the mirror of the mesh table as the restored state has it
    rc = refresh_mirror(p);
    if (!rc) rc = check(p, cudaStreamSynchronize(p->stream), "autotune");
    if (tile_out) *tile_out = best_tile;
    if (mode_out) *mode_out = best_mode;
    if (ms_out) *ms_out = best / steps;
    return rc;
}

int femstep_pool_set_schedule(femstep_pool* p, int tile, int mode) {
    if (!p) return fail(p, FEMSTEP_EINVAL, "null pool");
    if (p->in_flight) return fail(p, FEMSTEP_ESTATE, "a chunk is running: wait for it first");
    if (tile != 128 && tile != 256 && tile != 512) return fail(p, FEMSTEP_EINVAL, "tile must be 128, 256 or 512");
    if (!valid_mode(mode)) return fail(p, FEMSTEP_EINVAL, "bad mode");
    if (mode == FEMSTEP_POOL_GRAPH_TILED && tile != 128)
        return fail(p, FEMSTEP_EINVAL, "the tiled schedule runs tiles of 128");
    if (mode == FEMSTEP_POOL_GRAPH_STAGED && tile == 512)
        return fail(p, FEMSTEP_EINVAL, "the staged element pass runs tiles of 128 or 256");
    if (tile != p->tile) {
        // the instantaneous partials of the old tiling are stale
        cudaMemsetAsync(p->d.e_strain, 0, (size_t)p->part_cap * 8, p->stream);
        cudaMemsetAsync(p->d.n_kin, 0, (size_t)p->part_cap * 8, p->stream);
        p->dirty = true;
    }
    p->tile = tile;
    p->mode = mode;
    return check(p, cudaGetLastError(), "schedule");
}

int femstep_pool_profile(femstep_pool* p, int steps, double out[2]) {
    if (!p || !out || steps <= 0) return fail(p, FEMSTEP_EINVAL, "bad argument");
    if (p->broken) return fail(p, FEMSTEP_ESTATE, "the pool stopped after a device wait gave up");
    if (p->in_flight) return fail(p, FEMSTEP_ESTATE, "a chunk is running: wait for it first");
    int rc = rebuild(p);
    if (rc) return rc;
    const bool tiled = p->mode == FEMSTEP_POOL_GRAPH_TILED;
    if (tiled) rc = ensure_tiled(p);
    if (rc) return rc;
    PoolDevice dn = p->d;
    if (tiled) dn.offset = const_cast<uint32_t*>(p->d.part_off);
    cudaEvent_t ev[3];
    for (auto& e : ev) cudaEventCreate(&e);
    double te = 0.0, tn = 0.0;
    for (int s = 0; s < steps && !rc; ++s) {
        cudaEventRecord(ev[0], p->stream);
        if (tiled)
            fs::launch_pool_tiled_element_pass(p->d, s, p->stream);
        else
            fs::launch_pool_element_pass(p->d, p->tile, s, p->stream, p->mode == FEMSTEP_POOL_GRAPH_STAGED);
        cudaEventRecord(ev[1], p->stream);
        fs::launch_pool_node_pass(dn, p->tile, s, p->stream);
        cudaEventRecord(ev[2], p->stream);
        rc = check(p, cudaEventSynchronize(ev[2]), "profile");
        float a = 0.0f, b = 0.0f;
        cudaEventElapsedTime(&a, ev[0], ev[1]);
        cudaEventElapsedTime(&b, ev[1], ev[2]);
        te += a;
        tn += b;
    }
    if (!rc) {
        fs::launch_pool_advance(p->d, steps, p->stream);
        rc = refresh_mirror(p);
        if (!rc) rc = check(p, cudaStreamSynchronize(p->stream), "profile");
    }
    for (auto& e : ev) cudaEventDestroy(e);
    out[0] = te / steps;
    out[1] = tn / steps;
    return rc;
}

int femstep_pool_info(femstep_pool* p, long long out[8]) {
    if (!p || !out) return fail(p, FEMSTEP_EINVAL, "null argument");
    long long t = 0, n = 0, k = 0;
    for (const HostMesh& m : p->meshes)
        if (m.used) {
            t += m.T;
            n += m.N;
            ++k;
        }
    out[0] = t;
    out[1] = n;
    out[2] = k;
    out[3] = p->tile;
    out[4] = p->mode;
    out[5] = p->launches;
    // the pool's own arrays, and the tiled schedule's tables where they were built
    out[6] = (long long)(p->arena.bytes() + p->tiled.fixed_bytes + p->tiled.entries_cap * 10);
    out[7] = (long long)p->staging.count();
    return FEMSTEP_OK;
}

const char* femstep_pool_error(const femstep_pool* p) { return p ? p->error.c_str() : fs::last_error(); }

void femstep_pool_destroy(femstep_pool* p) {
    if (!p) return;
    if (p->stream) cudaStreamSynchronize(p->stream);
    drop_graph(p);
    free_tiled(p);
    p->arena.release();
    p->staging.release();
    if (p->h_meshes) cudaFreeHost(p->h_meshes);
    if (p->h_error) cudaFreeHost(p->h_error);
    if (p->ev0) cudaEventDestroy(p->ev0);
    if (p->ev1) cudaEventDestroy(p->ev1);
    if (p->stream) cudaStreamDestroy(p->stream);
    delete p;
}

}  // extern "C"
