// solver_api.cu -- host runtime of libmlmq_b200.so: device graphs, the solver
// context (distance array + queue workspace + persistent launch), the
// reference-compatible entry points and the one-shot host-buffer call.
#include "device_common.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_segmented_sort.cuh>
#include "mlmq_b200.h"
#include "mlmq_queue.cuh"
#include "sssp_plain.h"
#include "solver_internal.h"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

using namespace mlmq;

namespace mlmq {

int cuda_fail(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return MLMQ_OK;
    std::fprintf(stderr, "mlmq_b200: %s: %s\n", what, cudaGetErrorString(e));
    if (e == cudaErrorMemoryAllocation) return MLMQ_ERR_NOMEM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return MLMQ_ERR_NODEV;
    return MLMQ_ERR_CUDA;
}

namespace {

// One pool per device, created on first use.  A release threshold of "all"
// keeps freed blocks mapped for the next allocation of the process.
std::mutex g_pool_mu;
std::vector<cudaMemPool_t> g_pools;

int device_pool(cudaMemPool_t *out) {
    int dev = 0;
    int rc = cuda_fail(cudaGetDevice(&dev), "cudaGetDevice");
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if ((int)g_pools.size() <= dev) g_pools.resize((size_t)dev + 1, nullptr);
    if (!g_pools[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        rc = cuda_fail(cudaMemPoolCreate(&pool, &props), "cudaMemPoolCreate");
        if (rc) return rc;
        uint64_t keep = UINT64_MAX;
        rc = cuda_fail(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep),
                       "pool release threshold");
        if (rc) {
            cudaMemPoolDestroy(pool);
            return rc;
        }
        g_pools[dev] = pool;
    }
    *out = g_pools[dev];
    return MLMQ_OK;
}

// Page-locked copies of solver control blocks, carved from slabs of 64 that
// are kept for reuse: page-locking memory per solver costs more than the
// rest of creating one.
constexpr int CTL_SLAB = 64;
std::mutex g_pin_mu;
std::vector<unsigned *> g_pin_free;

}  // namespace

int pinned_ctl_alloc(unsigned **p) {
    std::lock_guard<std::mutex> lk(g_pin_mu);
    if (g_pin_free.empty()) {
        unsigned *slab = nullptr;
        const int rc = cuda_fail(cudaHostAlloc(&slab, sizeof(unsigned) * ctl::WORDS * CTL_SLAB,
                                               cudaHostAllocPortable),
                                 "pinned ctl");
        if (rc) return rc;
        for (int i = CTL_SLAB - 1; i >= 0; i--) g_pin_free.push_back(slab + (size_t)i * ctl::WORDS);
    }
    *p = g_pin_free.back();
    g_pin_free.pop_back();
    return MLMQ_OK;
}

void pinned_ctl_free(unsigned *p) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_pin_mu);
    g_pin_free.push_back(p);
}

namespace {
// Size classes of the pinned pool: powers of two from 4 KiB.
std::vector<std::vector<void *>> g_pinned_free(48);
int pinned_class(size_t bytes) {
    int c = 12;
    while (((size_t)1 << c) < bytes) c++;
    return c;
}
}  // namespace

int pinned_alloc(void **p, size_t bytes) {
    *p = nullptr;
    const int c = pinned_class(bytes ? bytes : 1);
    {
        std::lock_guard<std::mutex> lk(g_pin_mu);
        auto &fl = g_pinned_free[(size_t)c];
        if (!fl.empty()) {
            *p = fl.back();
            fl.pop_back();
            return MLMQ_OK;
        }
    }
    return cuda_fail(cudaHostAlloc(p, (size_t)1 << c, cudaHostAllocPortable | cudaHostAllocMapped),
                     "pinned host memory");
}

void pinned_free(const void *p, size_t bytes) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_pin_mu);
    g_pinned_free[(size_t)pinned_class(bytes ? bytes : 1)].push_back(const_cast<void *>(p));
}

int dev_alloc(void **p, size_t bytes, cudaStream_t st, const char *what) {
    *p = nullptr;
    cudaMemPool_t pool = nullptr;
    int rc = device_pool(&pool);
    if (rc) return rc;
    cudaError_t e = cudaMallocFromPoolAsync(p, bytes ? bytes : 1, pool, st);
    if (e == cudaErrorMemoryAllocation) {
        // The pool's free blocks may be too small or fragmented: give them
        // back to the driver and try once more.
        cudaGetLastError();
        cudaStreamSynchronize(st);
        cudaMemPoolTrimTo(pool, 0);
        e = cudaMallocFromPoolAsync(p, bytes ? bytes : 1, pool, st);
    }
    return cuda_fail(e, what);
}

void dev_free(const void *p, cudaStream_t st) {
    if (p) cudaFreeAsync(const_cast<void *>(p), st);
}

namespace {

__global__ void interleave_kernel(const int *__restrict__ col, const int *__restrict__ w, int2 *arcs,
                                  int64_t m) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x)
        arcs[i] = make_int2(col[i], w[i]);
}

// Largest out-degree of vertices [v0, v1) (out[0]) and largest weight of
// arcs [a0, a1) (out[1]).
__global__ void degree_weight_max_kernel(const int *__restrict__ row, int v0, int v1,
                                         const int *__restrict__ w, int64_t a0, int64_t a1, int *out) {
    int dmax = 0, wmax = 0;
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t v = v0 + tid; v < v1; v += stride) dmax = max(dmax, row[v + 1] - row[v]);
    for (int64_t e = a0 + tid; e < a1; e += stride) wmax = max(wmax, w[e]);
    dmax = __reduce_max_sync(FULL, dmax);
    wmax = __reduce_max_sync(FULL, wmax);
    if ((threadIdx.x & 31) == 0) {
        atomicMax(out, dmax);
        atomicMax(out + 1, wmax);
    }
}

// Radix-sort key of every arc: tail vertex in the high bits, weight in the
// low `wbits`, so one radix sort of all arcs orders them by vertex (keeping
// the CSR offsets valid) and by weight within a vertex.  One warp per vertex,
// lanes over its arcs, so a hub costs its degree / 32 steps.
// Keys of vertices [v0, v1); keys[i - a0] for arc i (a0 = row[v0]).
__global__ void arc_key_kernel(const int *__restrict__ row, int v0, int v1, int64_t a0,
                               const int *__restrict__ w, int wbits, unsigned long long *keys) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t v = v0 + warp; v < v1; v += nwarps) {
        const int b = row[v], e = row[v + 1];
        for (int i = b + lane; i < e; i += 32)
            keys[i - a0] = ((unsigned long long)v << wbits) | (unsigned)w[i];
    }
}

__global__ void interleave_keyed_kernel(const int *__restrict__ col, const unsigned long long *__restrict__ keys,
                                        unsigned long long wmask, int2 *arcs, int64_t m) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x)
        arcs[i] = make_int2(col[i], (int)(keys[i] & wmask));
}

// One 32-byte tile per vertex (layout in mlmq_queue.cuh): up to TILE_ARCS
// arcs inline, unused slots with dst -1; a vertex of higher degree holds
// {TILE_CSR, first arc, degree} instead.
__global__ void tile_kernel(const int *__restrict__ row, const int2 *__restrict__ arcs,
                            int4 *tiles, int n) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const int beg = row[v], deg = row[v + 1] - beg;
        int t[8] = {-1, 0, -1, 0, -1, 0, -1, 0};
        if (deg > TILE_ARCS) {
            t[0] = TILE_CSR;
            t[1] = beg;
            t[2] = deg;
        } else {
            for (int i = 0; i < deg; i++) {
                const int2 a = arcs[beg + i];
                t[2 * i] = a.x;
                t[2 * i + 1] = a.y;
            }
        }
        tiles[2 * (size_t)v] = make_int4(t[0], t[1], t[2], t[3]);
        tiles[2 * (size_t)v + 1] = make_int4(t[4], t[5], t[6], t[7]);
    }
}

// Wide tiles from the 32-byte ones: a vertex of at most TILE_ARCS_WIDE arcs
// gets them inline (its arcs in the same weight order), every other tile
// (CSR range, split vertex, piece) is copied with the extra slots empty.
__global__ void widen_tiles_kernel(const int4 *__restrict__ tiles, const int2 *__restrict__ arcs,
                                   int n, int slots, int4 *wide) {
    const int4 none = make_int4(-1, 0, -1, 0);
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < slots; v += gridDim.x * blockDim.x) {
        const int4 t0 = tiles[2 * (size_t)v], t1 = tiles[2 * (size_t)v + 1];
        int4 *o = wide + 4 * (size_t)v;
        if (v < n && t0.x == TILE_CSR && t0.z <= TILE_ARCS_WIDE) {
            const int beg = t0.y, deg = t0.z;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int2 a = 2 * q < deg ? arcs[beg + 2 * q] : make_int2(-1, 0);
                const int2 b = 2 * q + 1 < deg ? arcs[beg + 2 * q + 1] : make_int2(-1, 0);
                o[q] = make_int4(a.x, a.y, b.x, b.y);
            }
        } else {
            o[0] = t0;
            o[1] = (v < n && t0.x >= -1) ? t1 : none;  // inline arcs keep their second half
            o[2] = none;
            o[3] = none;
        }
    }
}

// Light arcs (weight < delta) of each vertex: a lower bound search in its
// weight-sorted arcs.
// Vertices of more than SPLIT_MIN arcs as {vertex, first arc, degree, 0}, in
// no particular order; *count may exceed cap only for invalid row offsets.
__global__ void heavy_kernel(const int *__restrict__ row, int n, int *count, int4 *out, int cap) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const int beg = row[v], deg = row[v + 1] - beg;
        if (deg > SPLIT_MIN) {
            const int k = atomicAdd(count, 1);
            if (k < cap) out[k] = make_int4(v, beg, deg, 0);
        }
    }
}

__global__ void light_split_kernel(const int *__restrict__ row, const int2 *__restrict__ arcs, int n,
                                   int delta, int *split) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        int lo = row[v], hi = row[v + 1];
        const int b = lo;
        while (lo < hi) {
            const int mid = lo + ((hi - lo) >> 1);
            if (arcs[mid].y < delta) lo = mid + 1;
            else hi = mid;
        }
        split[v] = lo - b;
    }
}

// Heavy vertices' tiles: {TILE_SPLIT, first piece, pieces, degree}.
__global__ void patch_tiles_kernel(const int *__restrict__ idx, const int4 *__restrict__ tile,
                                   int count, int4 *tiles) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) tiles[2 * (size_t)idx[i]] = tile[i];
}

__global__ void fill_kernel(int *p, int64_t n, int v) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        p[i] = v;
}

int ceil_log2(uint64_t x) {
    int l = 0;
    while ((1ull << l) < x) l++;
    return l;
}

}  // namespace

// L3 holds at most one record per vertex, and only reached vertices (at most
// m + 1 of them) push: its ring gets that many slots plus room for the pushes
// in flight, and at least 2^(MLMQ_MIN_RING_LOG2 + 1).
int l3_ring_log2(int64_t n, int64_t m) {
    const int64_t reach = std::min<int64_t>(n, m + 1);
    return std::min(30, std::max(MLMQ_MIN_RING_LOG2 + 1, ceil_log2((uint64_t)reach + (1u << 16))));
}

size_t l3_bits_bytes(int64_t n) { return sizeof(unsigned) * (size_t)((n + 31) / 32); }

namespace {

int env_int(const char *name, int dflt, bool *present) {
    const char *s = std::getenv(name);
    if (present) *present = s != nullptr;
    return s ? std::atoi(s) : dflt;
}

}  // namespace

int graph_light_split_cached(const mlmq_graph *gc, int delta, const int **out) {
    auto *g = const_cast<mlmq_graph *>(gc);
    std::lock_guard<std::mutex> lk(g->split_mu);
    for (auto &e : g->split_cache)
        if (e.first == delta) {
            *out = e.second;
            return MLMQ_OK;
        }
    return MLMQ_ERR_STATE;
}

int graph_light_split(const mlmq_graph *gc, int delta, const int **out) {
    auto *g = const_cast<mlmq_graph *>(gc);
    std::lock_guard<std::mutex> lk(g->split_mu);
    for (auto &e : g->split_cache)
        if (e.first == delta) {
            *out = e.second;
            return MLMQ_OK;
        }
    int *d = nullptr;
    int rc = dev_alloc(&d, sizeof(int) * (size_t)g->n, 0, "alloc(light split)");
    if (!rc) {
        const int blocks = (int)std::min<int64_t>(((int64_t)g->n + 255) / 256, 148 * 16);
        light_split_kernel<<<blocks, 256>>>(g->d_row, g->d_arcs, g->n, delta, d);
        rc = cuda_fail(cudaGetLastError(), "light split launch");
        // The legacy default stream does not wait for the library's
        // (non-blocking) solver, batch and server streams.
        if (!rc) rc = cuda_fail(cudaStreamSynchronize(0), "light split");
    }
    if (rc) {
        dev_free(d, 0);
        return rc;
    }
    g->split_cache.emplace_back(delta, d);
    *out = d;
    return MLMQ_OK;
}

int graph_tiles_cached(const mlmq_graph *gc, int vertex_tiles, const int4 **out, int *stride) {
    *out = nullptr;
    *stride = 2;
    if (vertex_tiles == 0) return MLMQ_OK;
    if (vertex_tiles == 1) {
        *out = gc->d_tiles;
        return MLMQ_OK;
    }
    auto *g = const_cast<mlmq_graph *>(gc);
    std::lock_guard<std::mutex> lk(g->split_mu);
    if (!g->d_tiles_wide) return MLMQ_ERR_STATE;
    *out = g->d_tiles_wide;
    *stride = 4;
    return MLMQ_OK;
}

int graph_tiles(const mlmq_graph *gc, int vertex_tiles, const int4 **out, int *stride) {
    if (vertex_tiles != 2) return graph_tiles_cached(gc, vertex_tiles, out, stride);
    auto *g = const_cast<mlmq_graph *>(gc);
    std::lock_guard<std::mutex> lk(g->split_mu);
    if (!g->d_tiles_wide) {
        int4 *d = nullptr;
        int rc = dev_alloc(&d, 4 * sizeof(int4) * (size_t)g->slots(), 0, "alloc(wide tiles)");
        if (!rc) {
            const int blocks = (int)std::min<int64_t>(((int64_t)g->slots() + 255) / 256, 148 * 16);
            widen_tiles_kernel<<<blocks, 256>>>(g->d_tiles, g->d_arcs, g->n, g->slots(), d);
            rc = cuda_fail(cudaGetLastError(), "wide tiles launch");
            if (!rc) rc = cuda_fail(cudaStreamSynchronize(0), "wide tiles");
        }
        if (rc) {
            dev_free(d, 0);
            return rc;
        }
        g->d_tiles_wide = d;
    }
    *out = g->d_tiles_wide;
    *stride = 4;
    return MLMQ_OK;
}

int fill_device(int *p, int64_t n, int v, cudaStream_t s) {
    if (n <= 0) return MLMQ_OK;
    int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
    fill_kernel<<<blocks, 256, 0, s>>>(p, n, v);
    return cuda_fail(cudaGetLastError(), "fill launch");
}

int validate_config(const mlmq_config &c) {
    if (c.queue_type != MLMQ_L1SLF_L2DQ && c.queue_type != MLMQ_L1V_L2DQ)
        return MLMQ_ERR_UNSUPPORTED;
    if (c.delta < 1 || c.bucket_num < 1 || c.bucket_num > NB_MAX - 1) return MLMQ_ERR_ARG;
    if (c.bucket_max < 1 || c.bucket_max > c.bucket_num) return MLMQ_ERR_ARG;
    if (c.l2_batch < 1 || c.l2_batch > 32 || c.min_read < 1 || c.min_read > 32) return MLMQ_ERR_ARG;
    if (c.large_degree < 1 || c.l1_spill < 1 || c.l1_spill > 32) return MLMQ_ERR_ARG;
    if (c.warps_per_block < 1 || c.warps_per_block > 31 || c.work_blocks < 0) return MLMQ_ERR_ARG;
    // Ring floor: pushes that passed the pressure check before a bucket's
    // pressure bit was set (at most 32 per warp, ~76K on a full B200) plus
    // claimed-but-unread slots must fit in the ring's free half, so a writer
    // never meets an unread record of the previous lap in practice.
    if (c.l2_cap_log2 != 0 && (c.l2_cap_log2 < MLMQ_MIN_RING_LOG2 || c.l2_cap_log2 > 28))
        return MLMQ_ERR_ARG;
    if (c.l3_cap_log2 != 0 && (c.l3_cap_log2 < MLMQ_MIN_RING_LOG2 || c.l3_cap_log2 > 30))
        return MLMQ_ERR_ARG;
    if (c.timeout_ms < 1) return MLMQ_ERR_ARG;
    if (c.l1_keep < 0 || c.l1_keep > c.l1_spill) return MLMQ_ERR_ARG;
    if (c.relax_precheck != 0 && c.relax_precheck != 1) return MLMQ_ERR_ARG;
    if (c.relax_unroll != 1 && c.relax_unroll != 2 && c.relax_unroll != 4) return MLMQ_ERR_ARG;
    if (c.relax_unroll > 1 && c.warps_per_block > MLMQ_MAX_UNROLLED_WARPS) return MLMQ_ERR_ARG;
    if (c.vertex_tiles < 0 || c.vertex_tiles > 2) return MLMQ_ERR_ARG;
    if (c.l1_ahead < 0) return MLMQ_ERR_ARG;
    if (c.topup < 0 || c.topup > 32) return MLMQ_ERR_ARG;
    if (c.bucket_sync != 0 && c.bucket_sync != 1) return MLMQ_ERR_ARG;
    if (c.light_heavy != 0 && c.light_heavy != 1) return MLMQ_ERR_ARG;
    if (c.light_heavy && !c.vertex_tiles) return MLMQ_ERR_ARG;
    return MLMQ_OK;
}

int status_to_error(unsigned st) {
    if (st & ST_QUEUE_FULL) return MLMQ_ERR_QUEUE_FULL;
    if (st & ST_TIMEOUT) return MLMQ_ERR_TIMEOUT;
    if (!(st & ST_DONE)) return MLMQ_ERR_STATE;
    if (st & ST_RANGE) return MLMQ_ERR_RANGE;
    return MLMQ_OK;
}

int device_sm_count(int *sms) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    // Two attribute queries (cudaGetDeviceProperties would fill in every
    // property, a cost paid on every solver creation).
    int major = 0, minor = 0, count = 0;
    e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
    if (major < 10) {
        std::fprintf(stderr, "mlmq_b200: device %d is sm_%d%d; this library is built for sm_100a\n",
                     dev, major, minor);
        return MLMQ_ERR_NODEV;
    }
    *sms = count;
    return MLMQ_OK;
}

}  // namespace mlmq

// ---------------------------------------------------------------------------
extern "C" const char *mlmq_strerror(int code) {
    switch (code) {
        case MLMQ_OK: return "ok";
        case MLMQ_ERR_CUDA: return "CUDA runtime error";
        case MLMQ_ERR_ARG: return "invalid argument";
        case MLMQ_ERR_TIMEOUT: return "device wait exceeded its time limit";
        case MLMQ_ERR_QUEUE_FULL: return "queue ring stayed full past its time limit";
        case MLMQ_ERR_STATE: return "call out of order or solve did not finish";
        case MLMQ_ERR_NOMEM: return "out of memory";
        case MLMQ_ERR_UNSUPPORTED: return "unsupported configuration";
        case MLMQ_ERR_RANGE: return "a distance sum reached INT_MAX";
        case MLMQ_ERR_IO: return "I/O or file format error";
        case MLMQ_ERR_NODEV: return "no sm_100 CUDA device";
        case MLMQ_ERR_BUSY: return "no free slot or device memory";
        case MLMQ_ERR_MISMATCH: return "distances differ from the caller's reference";
        default: return "unknown error";
    }
}

extern "C" int mlmq_config_default(mlmq_config *cfg) {
    if (!cfg) return MLMQ_ERR_ARG;
    std::memset(cfg, 0, sizeof(*cfg));
    // core/include/common.h:24-34, SS/SSSP/sssp.cuh:20, sssp_run.cu:895-896.
    cfg->queue_type = MLMQ_L1SLF_L2DQ;
    cfg->delta = 200000;
    cfg->work_blocks = 0;
    cfg->warps_per_block = 16;
    cfg->l2_batch = 8;
    cfg->bucket_num = 16;
    cfg->bucket_max = 4;
    cfg->min_read = 8;
    cfg->large_degree = 16;
    cfg->l1_spill = 32;
    cfg->l2_cap_log2 = 0;
    cfg->l3_cap_log2 = 0;
    cfg->timeout_ms = 20000;
    cfg->l1_keep = 0;
    cfg->relax_precheck = 1;
    cfg->relax_unroll = 4;
    cfg->l1_ahead = 4;
    cfg->vertex_tiles = 1;
    int rc = MLMQ_OK;
    bool have = false;
    int d = env_int("BENCH_DELTA", 200000, &have);
    if (have) {
        if (d <= 0) rc = MLMQ_ERR_ARG;
        else cfg->delta = d;
    }
    int wb = env_int("MLMQ_WORK_BLOCKS", 0, &have);
    if (have) {
        if (wb < 1) rc = MLMQ_ERR_ARG;
        else cfg->work_blocks = wb;
    }
    if (const char *qn = std::getenv("BENCH_QUEUE")) {
        if (std::strcmp(qn, "L1SLF_L2DQ") == 0) cfg->queue_type = MLMQ_L1SLF_L2DQ;
        else if (std::strcmp(qn, "L1V_L2DQ") == 0) cfg->queue_type = MLMQ_L1V_L2DQ;
        else rc = MLMQ_ERR_UNSUPPORTED;
    }
    return rc;
}

// ---- device graphs -----------------------------------------------------------

namespace {

// `h_row`: the same row offsets in host memory when the caller has them
// (saves copying them back to find the heavy vertices), else null.
// A vertex range [v0, v1) whose arcs [a0, a1) are sorted as one piece;
// `ready`, if set, is an event recorded once the range's destinations and
// weights (and the row offsets) are on the device.
struct ArcRange {
    int v0, v1;
    int64_t a0, a1;
    cudaEvent_t ready;
};

// Each vertex's arcs sorted by weight (light arcs, w < delta, then form a
// prefix for any delta) and interleaved into arcs[], range by range, on the
// legacy default stream.  A range whose largest vertex has more than
// SPLIT_MIN arcs is sorted with one radix sort of (vertex, weight) keys,
// which the skew of a power-law graph does not slow down; other ranges with
// a segmented sort, which suits small degrees.  Ranges let the upload sort
// one part of the graph while the next is still being copied (R-MAT-22
// upload 21.4 -> 14.7 ms, 9.8 ms of it the PCIe copy).
int build_arcs(int n, int64_t m, const int *d_row, const int *d_col, const int *d_w,
               const std::vector<ArcRange> &ranges, int2 *arcs) {
    int vbits = 1;
    while (vbits < 31 && ((n - 1) >> vbits) != 0) vbits++;
    int64_t max_arcs = 0;
    for (const ArcRange &r : ranges) max_arcs = std::max<int64_t>(max_arcs, r.a1 - r.a0);
    int *d_max = nullptr, *v_out = nullptr, *k32 = nullptr;
    unsigned long long *k_in = nullptr, *k_out = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    int rc = dev_alloc(&d_max, 2 * sizeof(int), 0, "alloc(max)");
    if (!rc) rc = dev_alloc(&v_out, sizeof(int) * (size_t)m, 0, "alloc(sort values)");
    for (size_t ri = 0; !rc && ri < ranges.size(); ri++) {
        const ArcRange &r = ranges[ri];
        if (r.a1 == r.a0) continue;
        if (r.ready) rc = cuda_fail(cudaStreamWaitEvent(0, r.ready, 0), "wait range");
        int maxes[2] = {0, 0};  // largest degree, largest weight in the range
        if (!rc) rc = cuda_fail(cudaMemsetAsync(d_max, 0, 2 * sizeof(int), 0), "max init");
        if (!rc) {
            const int blocks = (int)std::min<int64_t>((r.a1 - r.a0 + 255) / 256, 148 * 8);
            degree_weight_max_kernel<<<blocks, 256>>>(d_row, r.v0, r.v1, d_w, r.a0, r.a1, d_max);
            rc = cuda_fail(cudaGetLastError(), "max launch");
        }
        if (!rc) rc = cuda_fail(cudaMemcpy(maxes, d_max, sizeof(maxes), cudaMemcpyDeviceToHost),
                                "D2H max");
        const int cnt = (int)(r.a1 - r.a0);
        size_t need = 0;
        if (!rc && maxes[0] > SPLIT_MIN) {
            int wbits = 1;
            while (wbits < 31 && (maxes[1] >> wbits) != 0) wbits++;
            if (!k_in) rc = dev_alloc(&k_in, sizeof(unsigned long long) * (size_t)max_arcs, 0, "alloc(sort keys)");
            if (!rc && !k_out)
                rc = dev_alloc(&k_out, sizeof(unsigned long long) * (size_t)max_arcs, 0, "alloc(sort keys)");
            if (!rc)
                rc = cuda_fail(cub::DeviceRadixSort::SortPairs(nullptr, need, k_in, k_out, d_col + r.a0,
                                                               v_out + r.a0, cnt, 0, vbits + wbits),
                               "radix sort size");
            if (!rc && need > tmp_bytes) {
                dev_free(tmp, 0);
                tmp = nullptr;
                tmp_bytes = need;
                rc = dev_alloc(&tmp, tmp_bytes, 0, "alloc(sort)");
            }
            if (!rc) {
                const int blocks = (int)std::min<int64_t>(((int64_t)(r.v1 - r.v0) * 32 + 255) / 256, 148 * 16);
                arc_key_kernel<<<blocks, 256>>>(d_row, r.v0, r.v1, r.a0, d_w, wbits, k_in);
                rc = cuda_fail(cudaGetLastError(), "arc key launch");
            }
            size_t have = tmp_bytes;
            if (!rc)
                rc = cuda_fail(cub::DeviceRadixSort::SortPairs(tmp, have, k_in, k_out, d_col + r.a0,
                                                               v_out + r.a0, cnt, 0, vbits + wbits),
                               "radix sort arcs");
            if (!rc) {
                const int blocks = (int)std::min<int64_t>((cnt + 255) / 256, 148 * 16);
                interleave_keyed_kernel<<<blocks, 256>>>(v_out + r.a0, k_out, (1ull << wbits) - 1ull,
                                                         arcs + r.a0, cnt);
                rc = cuda_fail(cudaGetLastError(), "interleave launch");
            }
        } else if (!rc) {
            // Segments address the arrays by absolute arc index (the row
            // offsets), so the keys buffer spans all m arcs.
            if (!k32) rc = dev_alloc(&k32, sizeof(int) * (size_t)m, 0, "alloc(sort keys)");
            if (!rc)
                rc = cuda_fail(cub::DeviceSegmentedSort::SortPairs(nullptr, need, d_w, k32, d_col, v_out,
                                                                   (int)m, r.v1 - r.v0, d_row + r.v0,
                                                                   d_row + r.v0 + 1),
                               "sort size");
            if (!rc && need > tmp_bytes) {
                dev_free(tmp, 0);
                tmp = nullptr;
                tmp_bytes = need;
                rc = dev_alloc(&tmp, tmp_bytes, 0, "alloc(sort)");
            }
            size_t have = tmp_bytes;
            if (!rc)
                rc = cuda_fail(cub::DeviceSegmentedSort::SortPairs(tmp, have, d_w, k32, d_col, v_out,
                                                                   (int)m, r.v1 - r.v0, d_row + r.v0,
                                                                   d_row + r.v0 + 1),
                               "sort arcs");
            if (!rc) {
                const int blocks = (int)std::min<int64_t>((cnt + 255) / 256, 148 * 16);
                interleave_kernel<<<blocks, 256>>>(v_out + r.a0, k32 + r.a0, arcs + r.a0, cnt);
                rc = cuda_fail(cudaGetLastError(), "interleave launch");
            }
        }
    }
    dev_free(d_max, 0);
    dev_free(v_out, 0);
    dev_free(k32, 0);
    dev_free(k_in, 0);
    dev_free(k_out, 0);
    dev_free(tmp, 0);
    return rc;
}

int wrap_device(int n, int64_t m, const int *d_row, const int *d_col, const int *d_w,
                const std::vector<ArcRange> &ranges, mlmq_graph **out) {
    if (!out || n <= 0 || m < 0 || m >= INT_MAX || !d_row || (m > 0 && (!d_col || !d_w)))
        return MLMQ_ERR_ARG;
    auto *g = new (std::nothrow) mlmq_graph;
    if (!g) return MLMQ_ERR_NOMEM;
    g->n = n;
    g->m = m;
    g->d_row = const_cast<int *>(d_row);
    g->own_row = false;
    g->d_arcs = nullptr;
    // Everything below is ordered on the legacy default stream; the graph is
    // complete when this returns (one synchronisation of that stream at the
    // end; it does not wait for the library's non-blocking streams, so a
    // graph can be built while a server kernel runs).
    int rc = cuda_fail(cudaGetDevice(&g->device), "cudaGetDevice");
    if (!rc) rc = dev_alloc(&g->d_arcs, sizeof(int2) * (size_t)(m > 0 ? m : 1), 0, "alloc(arcs)");
    if (!rc && m > 0) rc = build_arcs(n, m, d_row, d_col, d_w, ranges, g->d_arcs);
    // Heavy vertices (more than SPLIT_MIN arcs) are found on the device; at
    // most m / (SPLIT_MIN + 1) exist.  Their pieces are laid out on the host
    // in vertex order.
    std::vector<int4> heavy_list;     // {vertex, first arc, degree, 0}
    if (!rc && m > SPLIT_MIN) {
        const int cap = (int)(m / (SPLIT_MIN + 1)) + 1;
        int *d_count = nullptr;
        int4 *d_list = nullptr;
        int count = 0;
        rc = dev_alloc(&d_count, sizeof(int), 0, "alloc(heavy count)");
        if (!rc) rc = dev_alloc(&d_list, sizeof(int4) * (size_t)cap, 0, "alloc(heavy list)");
        if (!rc) rc = cuda_fail(cudaMemsetAsync(d_count, 0, sizeof(int), 0), "heavy count");
        if (!rc) {
            const int blocks = (int)std::min<int64_t>(((int64_t)n + 255) / 256, 148 * 16);
            heavy_kernel<<<blocks, 256>>>(d_row, n, d_count, d_list, cap);
            rc = cuda_fail(cudaGetLastError(), "heavy launch");
        }
        if (!rc) rc = cuda_fail(cudaMemcpy(&count, d_count, sizeof(int), cudaMemcpyDeviceToHost),
                                "D2H heavy count");
        if (!rc && count > cap) rc = MLMQ_ERR_ARG;  // row offsets not monotone
        if (!rc && count > 0) {
            heavy_list.resize((size_t)count);
            rc = cuda_fail(cudaMemcpy(heavy_list.data(), d_list, sizeof(int4) * (size_t)count,
                                      cudaMemcpyDeviceToHost),
                           "D2H heavy list");
            std::sort(heavy_list.begin(), heavy_list.end(),
                      [](const int4 &x, const int4 &y) { return x.x < y.x; });
        }
        dev_free(d_count, 0);
        dev_free(d_list, 0);
    }
    std::vector<int> heavy;           // vertex ids
    std::vector<int4> piece_tiles;    // 2 per piece
    std::vector<int4> heavy_tiles;    // 1 per heavy vertex (first half of its tile)
    for (size_t h = 0; !rc && h < heavy_list.size(); h++) {
        const int v = heavy_list[h].x, beg = heavy_list[h].y, deg = heavy_list[h].z;
        const int np = (deg + PIECE_ARCS - 1) / PIECE_ARCS;
        if ((int64_t)n + g->pieces + np >= INT_MAX) {
            rc = MLMQ_ERR_RANGE;
            break;
        }
        heavy.push_back(v);
        heavy_tiles.push_back(make_int4(TILE_SPLIT, n + g->pieces, np, deg));
        for (int k = 0; k < np; k++) {
            const int b = beg + k * PIECE_ARCS;
            const int c = std::min(PIECE_ARCS, beg + deg - b);
            piece_tiles.push_back(make_int4(TILE_CSR, b, c, v));
            piece_tiles.push_back(make_int4(-1, 0, -1, 0));
        }
        g->pieces += np;
    }
    if (!rc) rc = dev_alloc(&g->d_tiles, 2 * sizeof(int4) * (size_t)g->slots(), 0, "alloc(tiles)");
    if (!rc) {
        int blocks = (int)std::min<int64_t>(((int64_t)n + 255) / 256, 148 * 16);
        tile_kernel<<<blocks, 256>>>(d_row, g->d_arcs, g->d_tiles, n);
        rc = cuda_fail(cudaGetLastError(), "tile launch");
    }
    if (!rc && g->pieces > 0) {
        rc = cuda_fail(cudaMemcpy(g->d_tiles + 2 * (size_t)n, piece_tiles.data(),
                                  sizeof(int4) * piece_tiles.size(), cudaMemcpyHostToDevice),
                       "H2D piece tiles");
        int *d_idx = nullptr;
        int4 *d_ht = nullptr;
        if (!rc) rc = dev_alloc(&d_idx, sizeof(int) * heavy.size(), 0, "alloc(heavy)");
        if (!rc) rc = dev_alloc(&d_ht, sizeof(int4) * heavy.size(), 0, "alloc(heavy tiles)");
        if (!rc) rc = cuda_fail(cudaMemcpy(d_idx, heavy.data(), sizeof(int) * heavy.size(),
                                           cudaMemcpyHostToDevice), "H2D heavy");
        if (!rc) rc = cuda_fail(cudaMemcpy(d_ht, heavy_tiles.data(), sizeof(int4) * heavy.size(),
                                           cudaMemcpyHostToDevice), "H2D heavy tiles");
        if (!rc) {
            const int hn = (int)heavy.size();
            patch_tiles_kernel<<<(hn + 255) / 256, 256>>>(d_idx, d_ht, hn, g->d_tiles);
            rc = cuda_fail(cudaGetLastError(), "patch launch");
        }
        dev_free(d_idx, 0);
        dev_free(d_ht, 0);
    }
    if (!rc) rc = cuda_fail(cudaStreamSynchronize(0), "graph build");
    if (rc) {
        cudaStreamSynchronize(0);
        mlmq_graph_free(g);
        return rc;
    }
    *out = g;
    return MLMQ_OK;
}

}  // namespace

extern "C" int mlmq_graph_wrap_device(int n, int64_t m, const int *d_row, const int *d_col,
                                      const int *d_w, mlmq_graph **out) {
    if (n <= 0 || m < 0) return MLMQ_ERR_ARG;
    return wrap_device(n, m, d_row, d_col, d_w, {ArcRange{0, n, 0, m, nullptr}}, out);
}

extern "C" int mlmq_graph_upload(int n, int64_t m, const int *row, const int *col, const int *w,
                                 mlmq_graph **out) {
    if (!out || n <= 0 || m < 0 || m >= INT_MAX || !row || (m > 0 && (!col || !w)))
        return MLMQ_ERR_ARG;
    if (row[0] != 0 || row[n] != m) return MLMQ_ERR_ARG;
    // The arcs go over in ranges of whole vertices, on a copy stream, and
    // each range is sorted as soon as it has arrived: the sort of one range
    // runs beside the copy of the next (a large graph: up to 8 ranges of
    // at least 4M arcs).
    std::vector<ArcRange> ranges;
    const int64_t parts = std::max<int64_t>(1, std::min<int64_t>(8, m / (4 << 20)));
    int v = 0;
    for (int64_t k = 1; k <= parts; k++) {
        const int64_t target = m * k / parts;
        const int v1 = k == parts ? n
                                  : (int)(std::upper_bound(row + v, row + n, target) - row) - 1;
        const int vend = std::max(v1, v);
        if (vend > v || k == parts) ranges.push_back(ArcRange{v, vend, row[v], row[vend], nullptr});
        v = vend;
    }
    int *d_row = nullptr, *d_col = nullptr, *d_w = nullptr;
    cudaStream_t cs = nullptr;
    int rc = dev_alloc(&d_row, sizeof(int) * ((size_t)n + 1), 0, "alloc(row)");
    if (!rc && m > 0) rc = dev_alloc(&d_col, sizeof(int) * (size_t)m, 0, "alloc(col)");
    if (!rc && m > 0) rc = dev_alloc(&d_w, sizeof(int) * (size_t)m, 0, "alloc(w)");
    // The copy stream starts after the allocations (ordered on stream 0).
    cudaEvent_t allocated = nullptr;
    if (!rc) rc = cuda_fail(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "copy stream");
    if (!rc) rc = cuda_fail(cudaEventCreateWithFlags(&allocated, cudaEventDisableTiming), "event");
    if (!rc) rc = cuda_fail(cudaEventRecord(allocated, 0), "event");
    if (!rc) rc = cuda_fail(cudaStreamWaitEvent(cs, allocated, 0), "event wait");
    if (!rc) rc = cuda_fail(cudaMemcpyAsync(d_row, row, sizeof(int) * ((size_t)n + 1),
                                            cudaMemcpyHostToDevice, cs), "H2D row");
    for (ArcRange &r : ranges) {
        if (rc || r.a1 == r.a0) continue;
        const size_t off = (size_t)r.a0, bytes = sizeof(int) * (size_t)(r.a1 - r.a0);
        rc = cuda_fail(cudaMemcpyAsync(d_col + off, col + off, bytes, cudaMemcpyHostToDevice, cs),
                       "H2D col");
        if (!rc) rc = cuda_fail(cudaMemcpyAsync(d_w + off, w + off, bytes, cudaMemcpyHostToDevice, cs),
                                "H2D w");
        if (!rc) rc = cuda_fail(cudaEventCreateWithFlags(&r.ready, cudaEventDisableTiming), "event");
        if (!rc) rc = cuda_fail(cudaEventRecord(r.ready, cs), "event");
    }
    // With no arcs the row offsets still have to arrive before the build.
    if (!rc && m == 0) rc = cuda_fail(cudaStreamSynchronize(cs), "H2D row");
    mlmq_graph *g = nullptr;
    if (!rc) rc = wrap_device(n, m, d_row, d_col, d_w, ranges, &g);
    if (cs) {
        cudaStreamSynchronize(cs);  // copies end before their buffers are freed
        cudaStreamDestroy(cs);
    }
    for (ArcRange &r : ranges)
        if (r.ready) cudaEventDestroy(r.ready);
    if (allocated) cudaEventDestroy(allocated);
    dev_free(d_col, 0);
    dev_free(d_w, 0);
    if (rc) {
        dev_free(d_row, 0);
        return rc;
    }
    g->own_row = true;
    *out = g;
    return MLMQ_OK;
}

extern "C" int mlmq_graph_prepare_light(const mlmq_graph *g, int delta) {
    if (!g || delta < 1) return MLMQ_ERR_ARG;
    const int *d = nullptr;
    return graph_light_split(g, delta, &d);
}

extern "C" int mlmq_graph_prepare_tiles(const mlmq_graph *g, int vertex_tiles) {
    if (!g || vertex_tiles < 0 || vertex_tiles > 2) return MLMQ_ERR_ARG;
    const int4 *t = nullptr;
    int stride = 0;
    return graph_tiles(g, vertex_tiles, &t, &stride);
}

extern "C" int mlmq_graph_pieces(const mlmq_graph *g, int *pieces) {
    if (!g || !pieces) return MLMQ_ERR_ARG;
    *pieces = g->pieces;
    return MLMQ_OK;
}

extern "C" int mlmq_graph_copy_arcs(const mlmq_graph *g, int *col, int *w) {
    if (!g || (g->m > 0 && (!col || !w))) return MLMQ_ERR_ARG;
    if (g->m == 0) return MLMQ_OK;
    std::vector<int2> arcs;
    try {
        arcs.resize((size_t)g->m);
    } catch (const std::bad_alloc &) {
        return MLMQ_ERR_NOMEM;
    }
    int rc = cuda_fail(cudaStreamSynchronize(0), "graph sync");
    if (!rc) rc = cuda_fail(cudaMemcpy(arcs.data(), g->d_arcs, sizeof(int2) * (size_t)g->m,
                                       cudaMemcpyDeviceToHost), "D2H arcs");
    if (rc) return rc;
    for (size_t i = 0; i < arcs.size(); i++) {
        col[i] = arcs[i].x;
        w[i] = arcs[i].y;
    }
    return MLMQ_OK;
}

extern "C" int mlmq_graph_size(const mlmq_graph *g, int *n, int64_t *m) {
    if (!g) return MLMQ_ERR_ARG;
    if (n) *n = g->n;
    if (m) *m = g->m;
    return MLMQ_OK;
}

namespace mlmq {

void graph_retain(const mlmq_graph *g) {
    if (g) const_cast<mlmq_graph *>(g)->refs.fetch_add(1, std::memory_order_relaxed);
}

void graph_release(const mlmq_graph *gc) {
    if (!gc) return;
    auto *g = const_cast<mlmq_graph *>(gc);
    if (g->refs.fetch_sub(1, std::memory_order_acq_rel) != 1) return;
    // Last reference: every solver, batch and served query that read the
    // graph has ended (each drops its reference only after its work is
    // done), so the memory goes back to the pool, stream-ordered, without
    // waiting for unrelated work on the device.
    dev_free(g->d_arcs, 0);
    dev_free(g->d_tiles, 0);
    dev_free(g->d_tiles_wide, 0);
    for (auto &e : g->split_cache) dev_free(e.second, 0);
    if (g->own_row) dev_free(g->d_row, 0);
    delete g;
}

}  // namespace mlmq

extern "C" void mlmq_graph_free(mlmq_graph *g) { graph_release(g); }

// ---- solver context ----------------------------------------------------------

extern "C" int mlmq_solver_create(const mlmq_graph *g, const mlmq_config *cfg_in,
                                  mlmq_solver **out) {
    if (!g || !out) return MLMQ_ERR_ARG;
    mlmq_config cfg;
    int rc = MLMQ_OK;
    if (cfg_in) cfg = *cfg_in;
    else if ((rc = mlmq_config_default(&cfg))) return rc;
    if ((rc = validate_config(cfg))) return rc;
    int sms = 0;
    if ((rc = device_sm_count(&sms))) return rc;

    auto *s = new (std::nothrow) mlmq_solver;
    if (!s) return MLMQ_ERR_NOMEM;
    graph_retain(g);  // dropped by mlmq_solver_destroy after its last launch
    s->g = g;
    s->cfg = cfg;
    s->device = g->device;
    const uint64_t m = (uint64_t)std::max<int64_t>(g->m, 1);
    s->l2_log = cfg.l2_cap_log2 ? cfg.l2_cap_log2
                                : std::min(24, std::max(MLMQ_MIN_RING_LOG2, ceil_log2(m / 2 + 1)));
    s->nids = g->slots() + (cfg.light_heavy ? g->n : 0);
    if (cfg.light_heavy && (rc = graph_light_split(g, cfg.delta, &s->split))) {
        mlmq_solver_destroy(s);
        return rc;
    }
    if ((rc = graph_tiles(g, cfg.vertex_tiles, &s->tiles, &s->tile_stride))) {
        mlmq_solver_destroy(s);
        return rc;
    }
    s->l3_log = cfg.l3_cap_log2 ? cfg.l3_cap_log2 : l3_ring_log2(s->nids, g->m);
    s->workers = cfg.warps_per_block;
    int bps = 0;
    rc = cuda_fail(plain_max_blocks_per_sm(s->workers, cfg.relax_unroll, &bps), "occupancy");
    if (!rc && bps < 1) rc = MLMQ_ERR_UNSUPPORTED;
    if (!rc) {
        const int maxgrid = bps * sms;
        s->grid = cfg.work_blocks > 0 ? std::min(cfg.work_blocks, maxgrid) : sms;
        if (s->grid > maxgrid) s->grid = maxgrid;
    }
    const size_t l2_bytes = sizeof(unsigned long long) * ((size_t)(cfg.bucket_num + 1) << s->l2_log);
    const size_t l3_bytes = sizeof(unsigned long long) * ((size_t)1 << s->l3_log);
    if (!rc) rc = cuda_fail(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "stream");
    if (!rc) rc = cuda_fail(cudaEventCreateWithFlags(&s->done, cudaEventDisableTiming), "event");
    if (!rc) rc = dev_alloc(&s->d_dist, sizeof(int) * (size_t)g->n, s->stream, "alloc(dist)");
    if (!rc) rc = dev_alloc(&s->d_l2, l2_bytes, s->stream, "alloc(L2)");
    if (!rc) rc = dev_alloc(&s->d_l3, l3_bytes, s->stream, "alloc(L3)");
    if (!rc) rc = dev_alloc(&s->d_l3bits, l3_bits_bytes(s->nids), s->stream, "alloc(L3 bits)");
    if (!rc) rc = dev_alloc(&s->d_ctl, sizeof(unsigned) * ctl::WORDS, s->stream, "alloc(ctl)");
    if (!rc) rc = pinned_ctl_alloc(&s->h_ctl);
    if (!rc) rc = fill_device(s->d_dist, g->n, INT_MAX, s->stream);
    if (!rc) rc = cuda_fail(cudaStreamSynchronize(s->stream), "solver init");
    if (rc) {
        mlmq_solver_destroy(s);
        return rc;
    }
    s->dirty = true;
    *out = s;
    return MLMQ_OK;
}

namespace mlmq {

// Makes the queue workspace clean: every ring slot empty, every counter 0.
static int reset_workspace(mlmq_solver *s, cudaStream_t st) {
    const size_t l2_bytes =
        sizeof(unsigned long long) * ((size_t)(s->cfg.bucket_num + 1) << s->l2_log);
    const size_t l3_bytes = sizeof(unsigned long long) * ((size_t)1 << s->l3_log);
    int rc = cuda_fail(cudaMemsetAsync(s->d_l2, 0xff, l2_bytes, st), "reset L2");
    if (!rc) rc = cuda_fail(cudaMemsetAsync(s->d_l3, 0xff, l3_bytes, st), "reset L3");
    if (!rc) rc = cuda_fail(cudaMemsetAsync(s->d_ctl, 0, sizeof(unsigned) * ctl::WORDS, st), "reset ctl");
    if (!rc) s->dirty = false;
    return rc;
}

}  // namespace mlmq

extern "C" int mlmq_solver_launch(mlmq_solver *s, int src, void *stream) {
    if (!s) return MLMQ_ERR_ARG;
    if (src < 0 || src >= s->g->n) return MLMQ_ERR_ARG;
    // A launch still outstanding (possibly on another stream) uses the same
    // workspace: it ends first; its status is superseded by this launch's.
    if (s->launched) {
        s->launched = false;
        if (cudaEventSynchronize(s->done) != cudaSuccess) {
            cudaGetLastError();
            s->dirty = true;
        }
    }
    cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
    int rc = MLMQ_OK;
    if (s->dirty && (rc = reset_workspace(s, st))) return rc;
    PlainParams p;
    p.n = s->g->n;
    p.nslots = s->g->slots();
    p.nids = s->nids;
    p.row = s->g->d_row;
    p.arcs = s->g->d_arcs;
    p.tiles = s->tiles;
    p.tile_stride = s->tile_stride;
    p.col = nullptr;
    p.w = nullptr;
    p.dist = s->d_dist;
    p.src = src;
    p.l2 = s->d_l2;
    p.l3 = s->d_l3;
    p.l3bits = s->d_l3bits;
    p.ctlw = s->d_ctl;
    p.nb = s->cfg.bucket_num;
    p.bm = s->cfg.bucket_max;
    p.batch = s->cfg.l2_batch;
    p.min_read = s->cfg.min_read;
    p.large = s->cfg.large_degree;
    p.l1_spill = s->cfg.l1_spill;
    p.l1_vector = s->cfg.queue_type == MLMQ_L1V_L2DQ;
    p.l1_keep = s->cfg.l1_keep;
    p.l1_ahead = s->cfg.l1_ahead;
    p.topup = s->cfg.topup;
    p.bucket_sync = s->cfg.bucket_sync;
    p.split = s->split;
    p.precheck = s->cfg.relax_precheck;
    p.delta = (unsigned)s->cfg.delta;
    p.l2_log = s->l2_log;
    p.l3_log = s->l3_log;
    p.workers = s->workers;
    p.timeout_ns = (unsigned long long)s->cfg.timeout_ms * 1000000ull;
    rc = cuda_fail(plain_launch(p, s->cfg.relax_unroll, s->grid, st), "persistent launch");
    if (rc) {
        s->dirty = true;
        return rc;
    }
    rc = cuda_fail(cudaMemcpyAsync(s->h_ctl, s->d_ctl, sizeof(unsigned) * ctl::WORDS,
                                   cudaMemcpyDeviceToHost, st), "status copy");
    if (!rc) rc = cuda_fail(cudaEventRecord(s->done, st), "event record");
    s->launched = !rc;
    if (rc) s->dirty = true;
    return rc;
}

extern "C" int mlmq_solver_wait(mlmq_solver *s) {
    if (!s) return MLMQ_ERR_ARG;
    if (!s->launched) return MLMQ_ERR_STATE;
    int rc = cuda_fail(cudaEventSynchronize(s->done), "solve");
    s->launched = false;
    if (rc) {
        s->dirty = true;
        return rc;
    }
    const unsigned st = s->h_ctl[ctl::STATUS];
    rc = status_to_error(st);
    if (rc && rc != MLMQ_ERR_RANGE) s->dirty = true;
    return rc;
}

extern "C" int mlmq_solver_solve(mlmq_solver *s, int src) {
    int rc = mlmq_solver_launch(s, src, nullptr);
    return rc ? rc : mlmq_solver_wait(s);
}

extern "C" int mlmq_solver_dist(mlmq_solver *s, int **d_dist) {
    if (!s || !d_dist) return MLMQ_ERR_ARG;
    *d_dist = s->d_dist;
    return MLMQ_OK;
}

extern "C" int mlmq_solver_copy_dist(mlmq_solver *s, int *h_dist) {
    if (!s || !h_dist) return MLMQ_ERR_ARG;
    int rc = cuda_fail(cudaMemcpyAsync(h_dist, s->d_dist, sizeof(int) * (size_t)s->g->n,
                                       cudaMemcpyDeviceToHost, s->stream), "D2H dist");
    if (!rc) rc = cuda_fail(cudaStreamSynchronize(s->stream), "D2H dist sync");
    return rc;
}

extern "C" int mlmq_solver_stats(mlmq_solver *s, mlmq_solve_stats *st) {
    if (!s || !st) return MLMQ_ERR_ARG;
    const unsigned long long *c = reinterpret_cast<const unsigned long long *>(s->h_ctl + ctl::STATS);
    st->pushed = c[ctl::ST_PUSHED];
    st->l3_pushed = c[ctl::ST_L3_PUSHED];
    st->relaxed = c[ctl::ST_RELAXED];
    st->improved = c[ctl::ST_IMPROVED];
    st->first_max = (uint32_t)c[ctl::ST_FIRST_MAX];
    st->batches = c[ctl::ST_BATCHES];
    st->idle = c[ctl::ST_IDLE];
    st->grid = s->grid;
    st->block = 32 * (s->workers + 1);
    st->status = s->h_ctl[ctl::STATUS];
    return MLMQ_OK;
}

extern "C" void mlmq_solver_destroy(mlmq_solver *s) {
    if (!s) return;
    // The last launch may have gone to a caller's stream: it ends before the
    // workspace goes back to the pool.
    if (s->done) cudaEventSynchronize(s->done);
    if (s->stream) cudaStreamSynchronize(s->stream);
    dev_free(s->d_dist, s->stream);
    dev_free(s->d_l2, s->stream);
    dev_free(s->d_l3, s->stream);
    dev_free(s->d_l3bits, s->stream);
    dev_free(s->d_ctl, s->stream);
    pinned_ctl_free(s->h_ctl);
    if (s->done) cudaEventDestroy(s->done);
    if (s->stream) cudaStreamDestroy(s->stream);
    graph_release(s->g);
    delete s;
}

extern "C" int mlmq_release_cached(void) {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    int rc = MLMQ_OK;
    for (cudaMemPool_t pool : g_pools)
        if (pool && !rc) rc = cuda_fail(cudaMemPoolTrimTo(pool, 0), "cudaMemPoolTrimTo");
    return rc;
}

extern "C" int mlmq_solve_host(int n, int64_t m, const int *row, const int *col, const int *w,
                               int nsrc, const int *srcs, int *h_dist, const mlmq_config *cfg) {
    if (nsrc < 0 || (nsrc > 0 && (!srcs || !h_dist))) return MLMQ_ERR_ARG;
    for (int k = 0; k < nsrc; k++)
        if (srcs[k] < 0 || srcs[k] >= n) return MLMQ_ERR_ARG;
    mlmq_graph *g = nullptr;
    int rc = mlmq_graph_upload(n, m, row, col, w, &g);
    if (rc) return rc;
    mlmq_solver *s = nullptr;
    rc = mlmq_solver_create(g, cfg, &s);
    // Two distance arrays: source k + 1 is solved into one while source k's
    // distances are copied out of the other (copy engines, beside the
    // persistent kernel).  The kernel's prologue initialises its array.
    int *own = s ? s->d_dist : nullptr, *spare = nullptr;
    if (!rc && nsrc > 1) rc = dev_alloc(&spare, sizeof(int) * (size_t)n, s->stream, "alloc(dist)");
    if (!rc && nsrc > 0) rc = mlmq_solver_launch(s, srcs[0], nullptr);
    for (int k = 0; !rc && k < nsrc; k++) {
        rc = mlmq_solver_wait(s);
        int *solved = s->d_dist;
        if (!rc && k + 1 < nsrc) {
            s->d_dist = solved == own ? spare : own;
            rc = mlmq_solver_launch(s, srcs[k + 1], nullptr);
        }
        if (!rc)
            rc = cuda_fail(cudaMemcpy(h_dist + (size_t)k * (size_t)n, solved, sizeof(int) * (size_t)n,
                                      cudaMemcpyDeviceToHost),
                           "D2H dist");
    }
    if (s) s->d_dist = own;
    mlmq_solver_destroy(s);  // waits for a launch still in flight after an error
    dev_free(spare, 0);
    mlmq_graph_free(g);
    return rc;
}

// ---- reference entry points ---------------------------------------------------
// Reference semantics (SS/SSSP/sssp_run.cu): one global, non-reentrant solver
// bound to a caller-owned device CSR.

// The reference's CLI (SS/SSSP/main.cu:19) defines this array of CPU-oracle
// distances; when the library is linked into that program the BENCH lines
// report correct=0/1 against it, as sssp_run.cu:849-853 does.
extern int *node_data_base __attribute__((weak));

namespace {
std::mutex g_mu;
mlmq_graph *g_graph = nullptr;
mlmq_solver *g_solver = nullptr;

double wall_ms() {
    return std::chrono::duration<double, std::milli>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}
}  // namespace

namespace mlmq {

int dropin_init(int m, int nnz, int *RowPtr, int *ColIdx, int *edge_data) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_solver) mlmq_solver_destroy(g_solver);
    if (g_graph) mlmq_graph_free(g_graph);
    g_solver = nullptr;
    g_graph = nullptr;
    int rc = mlmq_graph_wrap_device(m, nnz, RowPtr, ColIdx, edge_data, &g_graph);
    mlmq_config cfg;
    int crc = mlmq_config_default(&cfg);
    if (!rc && crc == MLMQ_ERR_UNSUPPORTED) rc = crc;
    if (!rc) rc = mlmq_solver_create(g_graph, &cfg, &g_solver);
    return rc;
}

int dropin_re_init() {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_solver) return MLMQ_ERR_STATE;
    int rc = fill_device(g_solver->d_dist, g_solver->g->n, INT_MAX, g_solver->stream);
    if (!rc) rc = cuda_fail(cudaStreamSynchronize(g_solver->stream), "re_init");
    return rc;
}

int dropin_run(int src) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_solver) return MLMQ_ERR_STATE;
    mlmq_config cfg;
    int rc = mlmq_config_default(&cfg);
    if (rc) return rc;
    if (std::memcmp(&cfg, &g_solver->cfg, sizeof(cfg)) != 0) {
        mlmq_solver *ns = nullptr;
        if ((rc = mlmq_solver_create(g_graph, &cfg, &ns))) return rc;
        mlmq_solver_destroy(g_solver);
        g_solver = ns;
    }
    if (src < 0 || src >= g_graph->n) return MLMQ_ERR_ARG;
    const char *qname = cfg.queue_type == MLMQ_L1V_L2DQ ? "L1V_L2DQ" : "L1SLF_L2DQ";
    std::printf("MLMQ_B200_CONFIG workers=%d blocks=%d delta=%d queue=%s\n",
                32 * g_solver->workers, g_solver->grid, cfg.delta, qname);
    const int warmups = env_int("BENCH_WARMUPS", 2, nullptr);
    const int repeats = env_int("BENCH_REPEATS", 3, nullptr);
    if (warmups < 0 || repeats < 1) return MLMQ_ERR_ARG;
    const int n = g_graph->n;
    std::vector<int> actual;
    int result = MLMQ_OK;
    for (int r = 0; r < warmups + repeats; r++) {
        const double q0 = wall_ms();
        const double s0 = wall_ms();
        rc = mlmq_solver_solve(g_solver, src);
        const double s1 = wall_ms();
        if (rc) return rc;
        int correct = -1;
        // A weak undefined variable has address NULL: test the address first.
        if (&node_data_base != nullptr && node_data_base != nullptr) {
            actual.resize((size_t)n);
            if ((rc = mlmq_solver_copy_dist(g_solver, actual.data()))) return rc;
            correct = std::memcmp(actual.data(), node_data_base, sizeof(int) * (size_t)n) == 0;
            if (!correct) result = MLMQ_ERR_MISMATCH;
        }
        const double q1 = wall_ms();
        std::printf("BENCH algorithm=MLMQ baseline=b200_sm100a gpu_count=1 source=%d repeat=%d "
                    "warmup=%d queue=%s solve_ms=%.6f query_wall_ms=%.6f correct=%d\n",
                    src, r, r < warmups, qname, s1 - s0, q1 - q0, correct);
        std::fflush(stdout);
    }
    return result;
}

int dropin_cp_data(int **node_data_h) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!node_data_h) return MLMQ_ERR_ARG;
    if (!g_solver) return MLMQ_ERR_STATE;
    int *h = (int *)std::malloc(sizeof(int) * (size_t)g_graph->n);
    if (!h) return MLMQ_ERR_NOMEM;
    int rc = mlmq_solver_copy_dist(g_solver, h);
    if (rc) {
        std::free(h);
        return rc;
    }
    *node_data_h = h;
    return MLMQ_OK;
}

}  // namespace mlmq

extern "C" int sssp_init(int m, int nnz, int *RowPtr, int *ColIdx, int *edge_data) {
    return mlmq::dropin_init(m, nnz, RowPtr, ColIdx, edge_data);
}
extern "C" int sssp_re_init(void) { return mlmq::dropin_re_init(); }
extern "C" int sssp_run_adaptive(int src, graph_info info) {
    (void)info;  // the reference ignores it too (adaptive setup is off, sssp_run.cu:894)
    return mlmq::dropin_run(src);
}
extern "C" int sssp_cp_data(int **node_data_h) { return mlmq::dropin_cp_data(node_data_h); }
