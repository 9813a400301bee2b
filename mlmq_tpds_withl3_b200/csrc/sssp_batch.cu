// sssp_batch.cu -- many single-source queries, on one or several graphs of
// uneven size, solved in ONE persistent launch.
//
// The reference's multi-source form is back-to-back full solver runs, one per
// source (SSSP/main.cu:213-307, run_multi_source_batch).  Here a launch hosts
// `nq` query slots.  Slot s is served by a contiguous group of CTAs
// (CTA c belongs to slot floor(c * nq / grid)); each slot owns its distance
// array, its L2/L3 rings and its control block, so every slot runs the
// single-source algorithm of sssp_plain_body.cuh unchanged -- its own
// termination, its own `first` -- while all slots share the graph arrays.
// A road-like query is bound by the latency of its dependent relaxations,
// not by bandwidth; running the queries side by side fills the GPU with
// independent chains, which is where the batched throughput comes from.
// Queries on the same graph read the same CSR, so its lines are shared in L2.
//
// The launch (parameter upload, kernel, status download) can be captured in
// a CUDA graph and replayed (mlmq_batch_run with use_graph = 1).
#include "mlmq_b200.h"
#include "solver_internal.h"
#include "sssp_plain.h"
// Per-warp counters in shared memory (see mlmq_queue.cuh).
#define MLMQ_WARP_STATS_SMEM 1
#include "sssp_plain_body.cuh"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

namespace mlmq {

constexpr int CTL_STRIDE = 512;  // words per slot control block (2 KiB, padded)

// What differs between the queries of a launch; everything else (queue
// configuration, per-slot workspace strides) is one kernel parameter, so it
// stays in the constant bank instead of occupying registers.
struct BatchQuery {
    const int *row;
    const int2 *arcs;
    const int4 *tiles;
    const int *split;
    int n, nslots, nids, src;
};
struct BatchParams {
    PlainParams base;  // configuration; dist/l2/l3/l3bits/ctlw point at slot 0's arrays
    const BatchQuery *__restrict__ queries;
    size_t dist_stride, l2_stride, l3_stride, bits_stride, ctl_stride;
    int nq;
};

// kSplit as for the single-solve kernel: true when a query's graph has
// pieces or the batch runs the light/heavy split.
template <int K, bool kSplit>
__global__ void __maxnreg__(SLOT_KERNEL_REGS) sssp_batch_kernel(BatchParams bp) {
    const unsigned g = gridDim.x;
    const unsigned nq = (unsigned)bp.nq;
    const unsigned s = (unsigned)(((unsigned long long)blockIdx.x * nq) / g);
    // First CTA of slot s: ceil(s * g / nq).
    const unsigned lo = (unsigned)(((unsigned long long)s * g + nq - 1) / nq);
    const unsigned hi = (unsigned)(((unsigned long long)(s + 1) * g + nq - 1) / nq);
    // The slot's parameters go to shared memory, not registers: the solve
    // reads them from there (or the constant bank), which keeps the kernel
    // at 56 registers, four CTAs of nine warps per SM.
    __shared__ PlainParams cta_params;
    if (threadIdx.x == 0) {
        PlainParams p = bp.base;
        const BatchQuery qy = bp.queries[s];
        p.row = qy.row;
        p.arcs = qy.arcs;
        p.tiles = qy.tiles;
        p.n = qy.n;
        p.nslots = qy.nslots;
        p.nids = qy.nids;
        p.split = qy.split;
        p.src = qy.src;
        p.dist = bp.base.dist + s * bp.dist_stride;
        p.l2 = bp.base.l2 + s * bp.l2_stride;
        p.l3 = bp.base.l3 + s * bp.l3_stride;
        p.l3bits = bp.base.l3bits + s * bp.bits_stride;
        p.ctlw = bp.base.ctlw + s * bp.ctl_stride;
        cta_params = p;
    }
    __syncthreads();
    plain_body<ArcsInterleaved, K, kSplit>(cta_params, blockIdx.x - lo, hi - lo);
}

const void *batch_kernel(int unroll, bool split) {
    switch (unroll) {
        case 1: return split ? (const void *)sssp_batch_kernel<1, true> : (const void *)sssp_batch_kernel<1, false>;
        case 2: return split ? (const void *)sssp_batch_kernel<2, true> : (const void *)sssp_batch_kernel<2, false>;
        default: return split ? (const void *)sssp_batch_kernel<4, true> : (const void *)sssp_batch_kernel<4, false>;
    }
}

}  // namespace mlmq

using namespace mlmq;

struct mlmq_batch {
    int device = 0;
    mlmq_config cfg{};
    int max_q = 0, max_n = 0;
    int grid = 0, workers = 0, l2_log = 0, l3_log = 0;
    int *d_dist = nullptr;            // max_q * max_n
    unsigned long long *d_l2 = nullptr;
    unsigned long long *d_l3 = nullptr;
    unsigned *d_l3bits = nullptr;     // max_q * bits_words
    size_t bits_words = 0;            // L3 vertex-bit words per slot
    unsigned *d_ctl = nullptr;        // max_q * CTL_STRIDE
    BatchQuery *d_queries = nullptr;  // max_q
    BatchQuery *h_queries = nullptr;  // pinned
    unsigned *h_ctl = nullptr;        // pinned copy of the control blocks
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    bool dirty = true, launched = false;
    int nq = 0;
    std::vector<int> n_of;            // vertex count per active slot
    cudaGraphExec_t exec = nullptr;   // captured launch of the current query set
    bool split = true;                // launch the split-capable kernel variant
    std::vector<long long> exec_key;  // (graph pointer, src) per slot of `exec`
    bool graph_cooperative = true;
    // Graphs referenced by the last launch and by `exec` (one reference
    // each): they stay allocated while a launch or a replay may read them,
    // and a freed graph's address cannot come back as a stale `exec_key`.
    std::vector<const mlmq_graph *> held;
};

namespace {

size_t l2_slots(const mlmq_batch *b) { return (size_t)(b->cfg.bucket_num + 1) << b->l2_log; }

int reset_all(mlmq_batch *b, cudaStream_t st) {
    int rc = cuda_fail(cudaMemsetAsync(b->d_l2, 0xff, sizeof(unsigned long long) * l2_slots(b) * b->max_q, st),
                       "batch reset L2");
    if (!rc) rc = cuda_fail(cudaMemsetAsync(b->d_l3, 0xff,
                                            sizeof(unsigned long long) * ((size_t)b->max_q << b->l3_log), st),
                            "batch reset L3");
    if (!rc) rc = cuda_fail(cudaMemsetAsync(b->d_ctl, 0, sizeof(unsigned) * CTL_STRIDE * b->max_q, st),
                            "batch reset ctl");
    if (!rc) b->dirty = false;
    return rc;
}

int enqueue(mlmq_batch *b, int nq, cudaStream_t st) {
    const int threads = 32 * (b->workers + 1);
    const size_t smem = plain_smem_bytes(b->workers);
    int rc = cuda_fail(cudaMemcpyAsync(b->d_queries, b->h_queries, sizeof(BatchQuery) * nq,
                                       cudaMemcpyHostToDevice, st), "batch queries");
    if (rc) return rc;
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3((unsigned)b->grid);
    lc.blockDim = dim3((unsigned)threads);
    lc.dynamicSmemBytes = smem;
    lc.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    lc.attrs = attr;
    lc.numAttrs = b->graph_cooperative ? 1 : 0;
    BatchParams bp{};
    PlainParams &p = bp.base;
    p.dist = b->d_dist;
    p.l2 = b->d_l2;
    p.l3 = b->d_l3;
    p.l3bits = b->d_l3bits;
    p.ctlw = b->d_ctl;
    p.nb = b->cfg.bucket_num;
    p.bm = b->cfg.bucket_max;
    p.batch = b->cfg.l2_batch;
    p.min_read = b->cfg.min_read;
    p.large = b->cfg.large_degree;
    p.l1_spill = b->cfg.l1_spill;
    p.l1_vector = b->cfg.queue_type == MLMQ_L1V_L2DQ;
    p.l1_keep = b->cfg.l1_keep;
    p.l1_ahead = b->cfg.l1_ahead;
    p.topup = b->cfg.topup;
    p.bucket_sync = b->cfg.bucket_sync;
    p.tile_stride = b->cfg.vertex_tiles == 2 ? 4 : 2;
    p.split = nullptr;  // per query
    p.precheck = b->cfg.relax_precheck;
    p.delta = (unsigned)b->cfg.delta;
    p.l2_log = b->l2_log;
    p.l3_log = b->l3_log;
    p.workers = b->workers;
    p.timeout_ns = (unsigned long long)b->cfg.timeout_ms * 1000000ull;
    bp.queries = b->d_queries;
    bp.dist_stride = (size_t)b->max_n;
    bp.l2_stride = l2_slots(b);
    bp.l3_stride = (size_t)1 << b->l3_log;
    bp.bits_stride = b->bits_words;
    bp.ctl_stride = CTL_STRIDE;
    bp.nq = nq;
    void *args[] = {&bp};
    rc = cuda_fail(cudaLaunchKernelExC(&lc, batch_kernel(b->cfg.relax_unroll, b->split), args),
                   "batch launch");
    if (rc) return rc;
    return cuda_fail(cudaMemcpyAsync(b->h_ctl, b->d_ctl, sizeof(unsigned) * CTL_STRIDE * nq,
                                     cudaMemcpyDeviceToHost, st), "batch status");
}

}  // namespace

extern "C" int mlmq_batch_create(int max_queries, int max_vertices, const mlmq_config *cfg_in,
                                 mlmq_batch **out) {
    if (!out || max_queries < 1 || max_vertices < 1) return MLMQ_ERR_ARG;
    mlmq_config cfg;
    int rc = MLMQ_OK;
    if (cfg_in) cfg = *cfg_in;
    else {
        if ((rc = mlmq_config_default(&cfg))) return rc;
        cfg.warps_per_block = 8;
    }
    if ((rc = validate_config(cfg))) return rc;
    if (cfg.warps_per_block > MLMQ_MAX_UNROLLED_WARPS) return MLMQ_ERR_ARG;
    int sms = 0;
    if ((rc = device_sm_count(&sms))) return rc;
    auto *b = new (std::nothrow) mlmq_batch;
    if (!b) return MLMQ_ERR_NOMEM;
    b->cfg = cfg;
    b->max_q = max_queries;
    b->max_n = max_vertices;
    b->workers = cfg.warps_per_block;
    b->l2_log = cfg.l2_cap_log2 ? cfg.l2_cap_log2 : MLMQ_MIN_RING_LOG2;
    b->l3_log = cfg.l3_cap_log2 ? cfg.l3_cap_log2 : l3_ring_log2(max_vertices, max_vertices);
    b->bits_words = l3_bits_bytes(max_vertices) / sizeof(unsigned);
    rc = cuda_fail(cudaGetDevice(&b->device), "cudaGetDevice");
    int bps = 0;
    if (!rc) {
        const int threads = 32 * (b->workers + 1);
        const size_t smem = plain_smem_bytes(b->workers);
        // The smaller occupancy of the two variants (either may run on the grid).
        for (int split = 0; split < 2 && !rc; split++) {
            const void *k = batch_kernel(cfg.relax_unroll, split != 0);
            rc = cuda_fail(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)plain_smem_limit()), "batch smem");
            int bk = 0;
            if (!rc)
                rc = cuda_fail(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bk, k, threads, smem),
                               "batch occupancy");
            bps = split ? std::min(bps, bk) : bk;
        }
    }
    if (!rc) {
        const int maxgrid = bps * sms;
        b->grid = cfg.work_blocks > 0 ? std::min(cfg.work_blocks, maxgrid) : maxgrid;
        if (b->grid < max_queries) {
            std::fprintf(stderr, "mlmq_batch_create: %d query slots need at least one CTA each; "
                                 "at most %d CTAs fit\n", max_queries, b->grid);
            rc = MLMQ_ERR_RANGE;
        }
    }
    const size_t nq = (size_t)max_queries;
    if (!rc) rc = cuda_fail(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "stream");
    if (!rc) rc = cuda_fail(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming), "event");
    // Device memory from the stream-ordered pool and pinned memory from the
    // pinned pool: destroying a batch then never synchronises the device.
    if (!rc) rc = dev_alloc(&b->d_dist, sizeof(int) * nq * (size_t)max_vertices, b->stream, "batch dist");
    if (!rc) rc = dev_alloc(&b->d_l2, sizeof(unsigned long long) * l2_slots(b) * nq, b->stream, "batch L2");
    if (!rc) rc = dev_alloc(&b->d_l3, sizeof(unsigned long long) * (nq << b->l3_log), b->stream, "batch L3");
    if (!rc) rc = dev_alloc(&b->d_l3bits, sizeof(unsigned) * b->bits_words * nq, b->stream, "batch L3 bits");
    if (!rc) rc = dev_alloc(&b->d_ctl, sizeof(unsigned) * CTL_STRIDE * nq, b->stream, "batch ctl");
    if (!rc) rc = dev_alloc(&b->d_queries, sizeof(BatchQuery) * nq, b->stream, "batch queries");
    if (!rc) rc = pinned_alloc(&b->h_queries, sizeof(BatchQuery) * nq);
    if (!rc) rc = pinned_alloc(&b->h_ctl, sizeof(unsigned) * CTL_STRIDE * nq);
    if (!rc) rc = reset_all(b, b->stream);
    if (!rc) rc = cuda_fail(cudaStreamSynchronize(b->stream), "batch init");
    if (rc) {
        mlmq_batch_destroy(b);
        return rc;
    }
    *out = b;
    return MLMQ_OK;
}

extern "C" int mlmq_batch_info(const mlmq_batch *b, int *grid, int *block, int *max_queries) {
    if (!b) return MLMQ_ERR_ARG;
    if (grid) *grid = b->grid;
    if (block) *block = 32 * (b->workers + 1);
    if (max_queries) *max_queries = b->max_q;
    return MLMQ_OK;
}

extern "C" int mlmq_batch_run(mlmq_batch *b, int nq, const mlmq_graph *const *graphs,
                              const int *srcs, int use_graph, void *stream) {
    if (!b || nq < 1 || nq > b->max_q || !graphs || !srcs) return MLMQ_ERR_ARG;
    for (int q = 0; q < nq; q++) {
        if (!graphs[q] || srcs[q] < 0 || srcs[q] >= graphs[q]->n ||
            graphs[q]->slots() + (b->cfg.light_heavy ? graphs[q]->n : 0) > b->max_n)
            return MLMQ_ERR_ARG;
        if (graphs[q]->device != b->device) return MLMQ_ERR_ARG;
    }
    // A launch still outstanding reads the pinned query table (its copy, or
    // a graph replay) and writes the workspace: it ends before either is
    // reused.  Its status is superseded by this launch's.
    if (b->launched) {
        b->launched = false;
        if (cudaEventSynchronize(b->done) != cudaSuccess) {
            cudaGetLastError();
            b->dirty = true;
        }
    }
    cudaStream_t st = stream ? (cudaStream_t)stream : b->stream;
    int rc = MLMQ_OK;
    if (b->dirty && (rc = reset_all(b, st))) return rc;
    // No launch of this batch is outstanding now: the graphs of this query
    // set replace the ones held for the previous one.
    std::vector<const mlmq_graph *> hold(graphs, graphs + nq);
    for (const mlmq_graph *g : hold) graph_retain(g);
    for (const mlmq_graph *g : b->held) graph_release(g);
    b->held.swap(hold);
    std::vector<long long> key;
    key.reserve(2 * (size_t)nq + 1);
    // The kernel variant is part of a captured launch: the split-capable one
    // when a graph has pieces or the light/heavy split is on.
    b->split = b->cfg.light_heavy != 0;
    for (int q = 0; q < nq; q++)
        if (graphs[q]->pieces > 0) b->split = true;
    key.push_back(b->split ? 1 : 0);
    b->n_of.assign((size_t)nq, 0);
    for (int q = 0; q < nq; q++) {
        const mlmq_graph *g = graphs[q];
        BatchQuery &qy = b->h_queries[q];
        qy.row = g->d_row;
        qy.arcs = g->d_arcs;
        int stride = 2;
        if ((rc = graph_tiles(g, b->cfg.vertex_tiles, &qy.tiles, &stride))) return rc;
        qy.n = g->n;
        qy.nslots = g->slots();
        qy.nids = g->slots() + (b->cfg.light_heavy ? g->n : 0);
        qy.split = nullptr;
        if (b->cfg.light_heavy && (rc = graph_light_split(g, b->cfg.delta, &qy.split))) return rc;
        qy.src = srcs[q];
        b->n_of[q] = g->n;
        key.push_back((long long)(uintptr_t)g);
        key.push_back(srcs[q]);
    }
    b->nq = nq;
    if (use_graph) {
        // Replay the captured launch when the query set is unchanged; the
        // parameters are read from the pinned host array at replay time.
        if (!b->exec || b->exec_key != key) {
            if (b->exec) {
                cudaGraphExecDestroy(b->exec);
                b->exec = nullptr;
            }
            cudaGraph_t graph = nullptr;
            for (int attempt = 0; attempt < 2 && !b->exec; attempt++) {
                rc = cuda_fail(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal),
                               "begin capture");
                if (rc) return rc;
                int erc = enqueue(b, nq, st);
                cudaError_t ce = cudaStreamEndCapture(st, &graph);
                if (erc == MLMQ_OK && ce == cudaSuccess) {
                    cudaError_t ie = cudaGraphInstantiate(&b->exec, graph, 0);
                    if (ie != cudaSuccess) b->exec = nullptr;
                }
                if (graph) cudaGraphDestroy(graph);
                graph = nullptr;
                cudaGetLastError();
                // Some drivers refuse cooperative kernels in graphs; the grid
                // never exceeds the occupancy limit, so a plain launch keeps
                // every CTA resident on an otherwise idle GPU.
                if (!b->exec) b->graph_cooperative = false;
            }
            if (!b->exec) return cuda_fail(cudaErrorNotSupported, "graph capture");
            b->exec_key = key;
        }
        rc = cuda_fail(cudaGraphLaunch(b->exec, st), "graph launch");
    } else {
        b->graph_cooperative = true;
        rc = enqueue(b, nq, st);
    }
    if (!rc) rc = cuda_fail(cudaEventRecord(b->done, st), "batch event");
    b->launched = !rc;
    if (rc) b->dirty = true;
    return rc;
}

extern "C" int mlmq_batch_wait(mlmq_batch *b) {
    if (!b) return MLMQ_ERR_ARG;
    if (!b->launched) return MLMQ_ERR_STATE;
    b->launched = false;
    int rc = cuda_fail(cudaEventSynchronize(b->done), "batch solve");
    if (rc) {
        b->dirty = true;
        return rc;
    }
    int worst = MLMQ_OK;
    for (int q = 0; q < b->nq; q++) {
        const int e = status_to_error(b->h_ctl[(size_t)q * CTL_STRIDE + ctl::STATUS]);
        if (e != MLMQ_OK && e != MLMQ_ERR_RANGE) b->dirty = true;
        if (e != MLMQ_OK && worst == MLMQ_OK) worst = e;
    }
    return worst;
}

extern "C" int mlmq_batch_query_status(const mlmq_batch *b, int q, unsigned *status,
                                       mlmq_solve_stats *st) {
    if (!b || q < 0 || q >= b->nq) return MLMQ_ERR_ARG;
    const unsigned *c = b->h_ctl + (size_t)q * CTL_STRIDE;
    if (status) *status = c[ctl::STATUS];
    if (st) {
        const unsigned long long *u = reinterpret_cast<const unsigned long long *>(c + ctl::STATS);
        st->pushed = u[ctl::ST_PUSHED];
        st->l3_pushed = u[ctl::ST_L3_PUSHED];
        st->relaxed = u[ctl::ST_RELAXED];
        st->improved = u[ctl::ST_IMPROVED];
        st->first_max = (uint32_t)u[ctl::ST_FIRST_MAX];
        st->batches = u[ctl::ST_BATCHES];
        st->idle = u[ctl::ST_IDLE];
        st->grid = b->grid;
        st->block = 32 * (b->workers + 1);
        st->status = c[ctl::STATUS];
    }
    return MLMQ_OK;
}

extern "C" int mlmq_batch_control(const mlmq_batch *b, int q, unsigned *words, int count) {
    if (!b || !words || q < 0 || q >= b->nq || count < 0 || count > CTL_STRIDE) return MLMQ_ERR_ARG;
    std::memcpy(words, b->h_ctl + (size_t)q * CTL_STRIDE, sizeof(unsigned) * (size_t)count);
    return MLMQ_OK;
}

extern "C" int mlmq_batch_dist(mlmq_batch *b, int q, int **d_dist) {
    if (!b || !d_dist || q < 0 || q >= b->max_q) return MLMQ_ERR_ARG;
    *d_dist = b->d_dist + (size_t)q * b->max_n;
    return MLMQ_OK;
}

extern "C" int mlmq_batch_copy_dist(mlmq_batch *b, int q, int *h_dist) {
    if (!b || !h_dist || q < 0 || q >= b->nq) return MLMQ_ERR_ARG;
    int rc = cuda_fail(cudaMemcpyAsync(h_dist, b->d_dist + (size_t)q * b->max_n,
                                       sizeof(int) * (size_t)b->n_of[q], cudaMemcpyDeviceToHost,
                                       b->stream), "batch D2H");
    if (!rc) rc = cuda_fail(cudaStreamSynchronize(b->stream), "batch D2H sync");
    return rc;
}

extern "C" void mlmq_batch_destroy(mlmq_batch *b) {
    if (!b) return;
    // The last launch may have gone to a caller's stream.
    if (b->launched && b->done) cudaEventSynchronize(b->done);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    const size_t nq = (size_t)b->max_q;
    dev_free(b->d_dist, b->stream);
    dev_free(b->d_l2, b->stream);
    dev_free(b->d_l3, b->stream);
    dev_free(b->d_l3bits, b->stream);
    dev_free(b->d_ctl, b->stream);
    dev_free(b->d_queries, b->stream);
    pinned_free(b->h_queries, sizeof(BatchQuery) * nq);
    pinned_free(b->h_ctl, sizeof(unsigned) * CTL_STRIDE * nq);
    for (const mlmq_graph *g : b->held) graph_release(g);
    if (b->done) cudaEventDestroy(b->done);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}
