// solver_internal.h -- library-private definitions shared by the host runtime
// translation units.
#pragma once

#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <mutex>
#include <utility>
#include <vector>

#include "mlmq_b200.h"

struct mlmq_graph {
    // References: the caller's handle (dropped by mlmq_graph_free) plus one
    // per solver, per batch query set and per served query that reads the
    // graph.  Its device memory goes back to the pool when the last one is
    // dropped, after the work that read it has ended -- never by a device-wide
    // synchronisation, which would wait for a running server kernel.
    std::atomic<int> refs{1};
    int n = 0;
    int64_t m = 0;
    int device = 0;
    int *d_row = nullptr;   // n + 1 row offsets (owned when own_row)
    bool own_row = false;
    int2 *d_arcs = nullptr; // m interleaved {dst, weight} (always owned)
    int4 *d_tiles = nullptr; // 2 per vertex and per piece: the vertex tiles (always owned)
    int pieces = 0;          // virtual vertices n .. n + pieces - 1 (split heavy vertices)
    int slots() const { return n + pieces; }
    // Per delta: light arcs (weight < delta) of each vertex, n ints.
    std::mutex split_mu;
    std::vector<std::pair<int, int *>> split_cache;
    // Wide tiles (4 per vertex and per piece, up to 8 arcs inline), built on
    // first use from d_tiles (guarded by split_mu).
    int4 *d_tiles_wide = nullptr;
};

struct mlmq_solver {
    const mlmq_graph *g = nullptr;
    mlmq_config cfg{};
    int device = 0;
    int grid = 0, workers = 0;
    int l2_log = 0, l3_log = 0;
    int nids = 0;               // queue ids: vertex slots, + n with the light/heavy split
    const int *split = nullptr; // light arcs per vertex for cfg.delta (owned by the graph)
    const int4 *tiles = nullptr; // tile array for cfg.vertex_tiles (owned by the graph)
    int tile_stride = 2;
    int *d_dist = nullptr;
    unsigned long long *d_l2 = nullptr;
    unsigned long long *d_l3 = nullptr;
    unsigned *d_l3bits = nullptr;  // one bit per vertex: the vertex has an L3 record
    unsigned *d_ctl = nullptr;
    unsigned *h_ctl = nullptr;  // pinned copy of the control block after each solve
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    bool dirty = true;          // queue workspace must be reset before the next launch
    bool launched = false;
};

namespace mlmq {

int cuda_fail(cudaError_t e, const char *what);
// Device buffers of graphs and solvers: from this device's stream-ordered
// pool (freed memory stays in the pool for reuse), ordered on `st`.
int dev_alloc(void **p, size_t bytes, cudaStream_t st, const char *what);
template <class T>
int dev_alloc(T **p, size_t bytes, cudaStream_t st, const char *what) {
    void *v = nullptr;
    const int rc = dev_alloc(&v, bytes, st, what);
    *p = static_cast<T *>(v);
    return rc;
}
void dev_free(const void *p, cudaStream_t st);
// One page-locked control-block copy (ctl::WORDS words) from a reused slab.
int pinned_ctl_alloc(unsigned **p);
void pinned_ctl_free(unsigned *p);
// Page-locked, device-mapped host memory from a process-wide pool of size
// classes.  Blocks go back to the pool, never to the driver: cudaFreeHost,
// like cudaFree, synchronises the device, and a batch or server freed while
// another server's persistent kernel runs must not wait for that kernel.
int pinned_alloc(void **p, size_t bytes);
template <class T>
int pinned_alloc(T **p, size_t bytes) {
    void *v = nullptr;
    const int rc = pinned_alloc(&v, bytes);
    *p = static_cast<T *>(v);
    return rc;
}
void pinned_free(const void *p, size_t bytes);
// Graph references (see mlmq_graph::refs).  graph_release frees the graph
// when it drops the last reference.
void graph_retain(const mlmq_graph *g);
void graph_release(const mlmq_graph *g);
int fill_device(int *p, int64_t n, int v, cudaStream_t s);
// Light arcs (weight < delta) of each vertex of g, computed once per delta
// and kept with the graph.
int graph_light_split(const mlmq_graph *g, int delta, const int **out);
// The same when already computed, else MLMQ_ERR_STATE (launches nothing).
int graph_light_split_cached(const mlmq_graph *g, int delta, const int **out);
// The tile array a configuration reads (vertex_tiles 1: d_tiles; 2: the
// wide tiles, built on first use; 0: none) and its int4 per tile.
int graph_tiles(const mlmq_graph *g, int vertex_tiles, const int4 **out, int *stride);
// The same without building anything (MLMQ_ERR_STATE if not built yet).
int graph_tiles_cached(const mlmq_graph *g, int vertex_tiles, const int4 **out, int *stride);
int validate_config(const mlmq_config &c);
int status_to_error(unsigned st);
int device_sm_count(int *sms);
// log2 of the L3 ring size for a graph of n vertices and m arcs.
int l3_ring_log2(int64_t n, int64_t m);
// Bytes of the per-vertex L3 bit array.
size_t l3_bits_bytes(int64_t n);

// Reference entry points; exported with C linkage (solver_api.cu) and with the
// reference's C++ linkage (drop_in.cpp).
int dropin_init(int m, int nnz, int *RowPtr, int *ColIdx, int *edge_data);
int dropin_re_init();
int dropin_run(int src);
int dropin_cp_data(int **node_data_h);

}  // namespace mlmq
