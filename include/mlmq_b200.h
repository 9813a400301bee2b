/*
 * mlmq_b200.h -- C ABI of libmlmq_b200.so, the B200 (sm_100a) delta-stepping
 * single-source shortest-path solver.
 *
 * Two groups of entry points:
 *
 *  1. The reference solver's own entry points, kept with the same names,
 *     argument meaning and index conventions so the library is a drop-in for
 *     the reference's single-GPU solver (hideoze/mlmq_tpds_withl3,
 *     evidence/l3_supplement_20260921_v2/single_source/SSSP/sssp_run.cu):
 *     sssp_init, sssp_re_init, sssp_run_adaptive, sssp_cp_data.  They are
 *     exported twice: with C linkage (declared here) and with the reference's
 *     C++ linkage (declared in sssp_drop_in.h) so the reference's own caller,
 *     SS/SSSP/main.cu, links against this library unchanged.
 *
 *  2. The library's own mlmq_* API: host graph generators and .gr I/O,
 *     device graphs, a re-entrant solver context, the batched multi-source
 *     solver and the serving loop.
 *
 * Conventions: vertex ids are 0-based; distances are int32 with INT_MAX
 * (0x7FFFFFFF) meaning unreachable, as in the reference (core/include/
 * common.h:11-20, VALUE_TYPE=int, DIST_MAX=INT_MAX); edge weights must be
 * non-negative and every finite distance must be < INT_MAX.  Every function
 * returns 0 on success or a negative MLMQ_ERR_* code; none calls exit().
 */
#ifndef MLMQ_B200_H
#define MLMQ_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error codes ------------------------------------------------------ */
#define MLMQ_OK 0
#define MLMQ_ERR_CUDA (-1)        /* a CUDA runtime call failed */
#define MLMQ_ERR_ARG (-2)         /* invalid argument */
#define MLMQ_ERR_TIMEOUT (-3)     /* a device-side wait ran past its limit */
#define MLMQ_ERR_QUEUE_FULL (-4)  /* a queue ring stayed full past its limit */
#define MLMQ_ERR_STATE (-5)       /* call out of order (e.g. run before init) */
#define MLMQ_ERR_NOMEM (-6)       /* host or device allocation failed */
#define MLMQ_ERR_UNSUPPORTED (-7) /* configuration not built in this library */
#define MLMQ_ERR_RANGE (-8)       /* a distance sum reached INT_MAX */
#define MLMQ_ERR_IO (-9)          /* file open/read/write or format error */
#define MLMQ_ERR_NODEV (-10)      /* no CUDA device, or not sm_100 */
#define MLMQ_ERR_BUSY (-11)       /* serving: no free slot or memory now */
#define MLMQ_ERR_MISMATCH (-12)   /* sssp_run_adaptive: result differs from the
                                     caller's CPU distances (node_data_base) */

/* Human-readable name of an MLMQ_ERR_* code. */
const char *mlmq_strerror(int code);

/* ---- queue configuration (reference: core/include/adaptive.h:5-62) ----- */

/* Queue types, numbered as the reference's enum mlmq_type
 * (core/include/common.h:85-108).  This library implements L1SLF_L2DQ (the
 * type the reference's timed path forces, sssp_run.cu:895) and L1V_L2DQ. */
#define MLMQ_L1V_L2DQ 0
#define MLMQ_L1SLF_L2DQ 19

/* Smallest queue ring (log2 slots) a configuration may ask for. */
#define MLMQ_MIN_RING_LOG2 18
/* Most worker warps per CTA when relax_unroll > 1 (plus one manager warp:
   800 threads); with relax_unroll 1 the limit is 31. */
#define MLMQ_MAX_UNROLLED_WARPS 24

typedef struct mlmq_config {
    int queue_type;      /* MLMQ_L1SLF_L2DQ (default) or MLMQ_L1V_L2DQ */
    int delta;           /* bucket width; reference BENCH_DELTA, default 200000 */
    int work_blocks;     /* persistent CTAs; 0 = one per SM that fits
                            (reference MLMQ_WORK_BLOCKS) */
    int warps_per_block; /* worker warps per CTA (reference: 512 threads = 16) */
    int l2_batch;        /* slots claimed per bucket read (l2_batch_size, 8) */
    int bucket_num;      /* L2 buckets (BNUM, 16; at most 32) */
    int bucket_max;      /* buckets readable at once (BUCKET_MAX, 4) */
    int min_read;        /* records wanted per read (MIN_READ_GRA, 8) */
    int large_degree;    /* warp-cooperative relaxation at this out-degree
                            (LARGEV, 16) */
    int l1_spill;        /* L1 spills to L2 when it holds more (32) */
    int l2_cap_log2;     /* log2 slots per L2 bucket ring; 0 = sized from graph;
                            else MLMQ_MIN_RING_LOG2..28 */
    int l3_cap_log2;     /* log2 slots of the L3 ring; 0 = sized from graph;
                            else MLMQ_MIN_RING_LOG2..30 */
    int timeout_ms;      /* device wait limit per solve (default 20000) */
    int l1_keep;         /* on a spill, records kept at the L1 front (0 = spill
                            all, the reference's rule; at most l1_spill) */
    int relax_precheck;  /* 1 (default): read dist[dst] first; a smaller
                            candidate is pushed and written with a
                            fire-and-forget min (red.min); 0: atomicMin
                            directly, its returned value decides the push */
    int relax_unroll;    /* rounds of 32 arcs a warp keeps in flight: 1, 2 or
                            4 (default 4; above 1 at most
                            MLMQ_MAX_UNROLLED_WARPS worker warps per CTA) */
    int l1_ahead;        /* a winner stays in the warp's L1 only while its
                            bucket is below first + l1_ahead, else it goes
                            to L2/L3 through the warp's outbox (default 4;
                            0: no limit, the reference's L1) */
    int topup;           /* a warp that takes fewer than `topup` records from
                            its L1 fills the rest of the warp from L2 in the
                            same iteration (default 0 = off: it lengthens a
                            single solve's critical path; batches use it) */
    int bucket_sync;     /* 1: the bucket window moves on only when no record
                            taken from the queues is still being worked on
                            (bulk-synchronous buckets): fewer redundant
                            relaxations where buckets are wide and few
                            (power-law graphs), slower where they are many
                            (grids); default 0 */
    int light_heavy;     /* 1: delta-stepping's light/heavy split: a record
                            relaxes its light arcs (weight < delta) at once
                            and its heavy arcs one bucket later, when its
                            distance is final, so heavy arcs are relaxed
                            about once; needs vertex tiles, and vertex slots
                            n + pieces + n in batches and servers; default 0 */
    int vertex_tiles;    /* 1 (default): read each vertex's adjacency from its
                            32-byte tile (up to 4 arcs inline, else its CSR
                            range); 2: 64-byte tiles with up to 8 arcs
                            inline (built on first use, kept with the graph);
                            0: row offsets, then arcs */
} mlmq_config;

/* Fills *cfg with the reference's defaults (common.h:24-34, sssp.cuh:20,
 * sssp_run.cu:896) and then applies the environment overrides the reference
 * reads: BENCH_DELTA, BENCH_QUEUE, MLMQ_WORK_BLOCKS. */
int mlmq_config_default(mlmq_config *cfg);

/* ---- 1. reference entry points (C linkage) ---------------------------- */

/* Layout-compatible with the reference's struct graph_info
 * (core/include/graph_info.h:8-22); passed by value, read-only. */
typedef struct graph_info {
    int m;
    int nnz;
    float avg_nnz;
    float max_nnz;
    float dev_nnz;
    float avg_weight;
    float dev_weight;
    float max_weight;
    float diameter;
} graph_info;

/* SS/SSSP/sssp_run.cu:676.  Binds a caller-owned DEVICE CSR: m vertices,
 * nnz arcs, RowPtr[m+1], ColIdx[nnz] (0-based), edge_data[nnz].  Allocates
 * the distance array and queue storage on the current device. */
int sssp_init(int m, int nnz, int *RowPtr, int *ColIdx, int *edge_data);
/* SS/SSSP/sssp_run.cu:709.  Resets every distance to INT_MAX. */
int sssp_re_init(void);
/* SS/SSSP/sssp_run.cu:888.  Solves from 0-based src with the configuration
 * of mlmq_config_default().  Like the reference it runs BENCH_WARMUPS (2)
 * untimed and BENCH_REPEATS (3) timed solves and prints one
 * "BENCH algorithm=MLMQ ..." line per solve. */
int sssp_run_adaptive(int src, graph_info info);
/* SS/SSSP/sssp_run.cu:749.  *node_data_h receives a malloc()ed host array of
 * m distances (0-based) that the caller frees. */
int sssp_cp_data(int **node_data_h);

/* ---- 2a. host graphs -------------------------------------------------- */

typedef struct mlmq_host_graph mlmq_host_graph;

/* width x height 4-neighbour grid, id = y*width + x; each undirected edge is
 * dropped with probability drop_p (seeded Bernoulli); both arcs share one
 * weight uniform in [wmin, wmax]. */
int mlmq_hgraph_grid(int width, int height, double drop_p, int wmin, int wmax,
                     uint64_t seed, mlmq_host_graph **out);
/* npoints uniform in the unit square joined to their k nearest neighbours,
 * symmetrised, weight = round(scale * euclid) + 1; vertex ids follow a
 * Morton order of a cell grid; perm[id] = index of the generated point. */
int mlmq_hgraph_knn(int npoints, int k, double scale, uint64_t seed,
                    mlmq_host_graph **out);
/* R-MAT: 2^scale vertices, edge_factor * 2^scale sampled directed arcs with
 * quadrant probabilities (a, b, c, 1-a-b-c); self-loops and duplicates
 * removed; weight uniform in [wmin, wmax]. */
int mlmq_hgraph_rmat(int scale, int edge_factor, double a, double b, double c,
                     int wmin, int wmax, uint64_t seed, mlmq_host_graph **out);
/* Copies a host CSR (validated like the reference exporter,
 * scripts/multigpu/supplement_graph.cpp:21-28). */
int mlmq_hgraph_from_csr(int n, int64_t m, const int *row, const int *col,
                         const int *w, mlmq_host_graph **out);
/* Galois/LonestarGPU .gr v1 (SSSP/csr_graph.cu:185-300, 302-418). */
int mlmq_hgraph_read_gr(const char *path, mlmq_host_graph **out);
int mlmq_hgraph_write_gr(const mlmq_host_graph *g, const char *path);
/* BFS locality reordering (graph_transform/reorder_gr.cu:96-190): new ids in
 * the discovery order of a queue BFS from root (arcs scanned in CSR order),
 * unreached vertices after them in ascending id; perm[new] = old,
 * invperm[old] = new (n entries each, may be NULL). */
int mlmq_hgraph_reorder_bfs(const mlmq_host_graph *g, int root, mlmq_host_graph **out,
                            int *perm, int *invperm);
/* The same reordering as a device preprocessing step (level-synchronous
 * search that reproduces the FIFO discovery order exactly): the CSR in
 * d_row/d_col/d_w (device, current device) is written reordered to
 * d_row_out[n+1], d_col_out[m], d_w_out[m], with d_perm[new] = old and
 * d_invperm[old] = new (n each), on `stream` (a cudaStream_t; NULL = legacy
 * default stream).  Temporary device memory comes from the library's pool.
 * Returns when the result is complete.  Output equals
 * mlmq_hgraph_reorder_bfs byte for byte. */
int mlmq_reorder_bfs_device(int n, int64_t m, const int *d_row, const int *d_col, const int *d_w,
                            int root, int *d_row_out, int *d_col_out, int *d_w_out, int *d_perm,
                            int *d_invperm, void *stream);
/* mlmq_hgraph_reorder_bfs computed on the current device: the host graph is
 * copied over, reordered by mlmq_reorder_bfs_device and copied back. */
int mlmq_hgraph_reorder_bfs_gpu(const mlmq_host_graph *g, int root, mlmq_host_graph **out,
                                int *perm, int *invperm);
/* Chain-shortcut augmentation G+ (SSSP/l3/l3_chain_shortcuts.h:23-109):
 * adds one arc per maximal walk through degree-2 chain vertices, keeps every
 * original arc, so distances are unchanged.  The output equals the reference
 * builder's byte for byte; the walks are resolved by pointer jumping.  cut = n places no partition
 * restriction; stats (may be NULL): chain vertices, shortcuts, longest walk,
 * walks dropped for INT_MAX overflow, arcs represented. */
int mlmq_hgraph_chain_shortcuts(const mlmq_host_graph *g, int cut, int source,
                                mlmq_host_graph **out, int64_t *stats);
/* Borrowed views; valid until mlmq_hgraph_free.  perm may be NULL. */
int mlmq_hgraph_view(const mlmq_host_graph *g, int *n, int64_t *m, const int **row,
                     const int **col, const int **w, const int **perm);
void mlmq_hgraph_free(mlmq_host_graph *g);

/* ---- 2b. device graphs and the solver context ------------------------- */

typedef struct mlmq_graph mlmq_graph;
typedef struct mlmq_solver mlmq_solver;

/* Device memory of graphs and solvers comes from a stream-ordered pool per
 * device that keeps freed memory for the next graph or solver (no release
 * threshold), so code that builds and drops them per call, as
 * mlmq_solve_host does, maps device memory once.  This returns the pools'
 * unused memory to the driver (e.g. before another allocator needs it);
 * memory still in use is not affected. */
int mlmq_release_cached(void);

/* Copies a host CSR to the current device and builds the interleaved
 * {dst, weight} arc array the kernels read (each vertex's arcs sorted by
 * weight), the vertex tiles and the pieces of split vertices; returns when
 * the graph is complete.  A large graph's arcs go over in ranges of whole
 * vertices on a copy stream of its own, each range sorted while the next is
 * copied; with page-locked host arrays the copies run at PCIe speed (the
 * driver stages pageable ones). */
int mlmq_graph_upload(int n, int64_t m, const int *row, const int *col, const int *w,
                      mlmq_graph **out);
/* Wraps a caller-owned device CSR (not copied; must outlive the graph). */
int mlmq_graph_wrap_device(int n, int64_t m, const int *d_row, const int *d_col,
                           const int *d_w, mlmq_graph **out);
int mlmq_graph_size(const mlmq_graph *g, int *n, int64_t *m);
/* Vertices of more than 1024 arcs are relaxed as pieces of at most 512 arcs
 * that different warps take in parallel; each piece is a virtual vertex id
 * after the graph's n.  A batch or server solving this graph needs
 * max_vertices >= n + pieces. */
int mlmq_graph_pieces(const mlmq_graph *g, int *pieces);
/* Computes (once, kept with the graph) each vertex's number of light arcs
 * (weight < delta) for the light/heavy split.  Solvers and batches do it on
 * first use; a server cannot, because its persistent launch holds every SM:
 * prepare every (graph, delta) its light_heavy queries use before creating
 * the server (mlmq_server_submit_cfg returns MLMQ_ERR_STATE otherwise).
 * Likewise bind graphs before a server starts on the same device. */
int mlmq_graph_prepare_light(const mlmq_graph *g, int delta);
/* Builds (once, kept with the graph) the tile array of a vertex_tiles
 * setting: only 2 (wide tiles) needs building; solvers and batches do it on
 * first use, a server cannot (as for mlmq_graph_prepare_light): prepare
 * before the server starts. */
int mlmq_graph_prepare_tiles(const mlmq_graph *g, int vertex_tiles);
/* Copies the graph's arcs, in the order the kernels read them (each vertex's
 * arcs a permutation of its input arcs, sorted by weight), into host arrays
 * of m ints: col[e] destination, w[e] weight.  Synchronous; for inspection
 * and tests. */
int mlmq_graph_copy_arcs(const mlmq_graph *g, int *col, int *w);
void mlmq_graph_free(mlmq_graph *g);

/* A solver owns one distance array and one queue workspace on the device
 * current at creation.  cfg may be NULL (mlmq_config_default). */
int mlmq_solver_create(const mlmq_graph *g, const mlmq_config *cfg, mlmq_solver **out);
/* Enqueues one complete solve from src on `stream` (a cudaStream_t; NULL =
 * the solver's own stream): distance reset, seed, persistent kernel.
 * Returns after the launch; mlmq_solver_wait reports the outcome.  A launch
 * while the previous one is outstanding waits for it first (they share the
 * workspace); the earlier outcome is then not reported. */
int mlmq_solver_launch(mlmq_solver *s, int src, void *stream);
/* Blocks until the last launch ends; returns its status as MLMQ_ERR_*. */
int mlmq_solver_wait(mlmq_solver *s);
/* launch + wait. */
int mlmq_solver_solve(mlmq_solver *s, int src);
/* Device pointer to the n distances of the last solve. */
int mlmq_solver_dist(mlmq_solver *s, int **d_dist);
/* Copies the n distances to host memory (synchronous). */
int mlmq_solver_copy_dist(mlmq_solver *s, int *h_dist);

typedef struct mlmq_solve_stats {
    uint64_t pushed;     /* records written to L2/L3 */
    uint64_t l3_pushed;  /* of which to the L3 ring */
    uint64_t relaxed;    /* arcs scanned */
    uint64_t improved;   /* successful atomicMin updates */
    uint32_t first_max;  /* last bucket index reached */
    int grid;            /* persistent CTAs launched */
    int block;           /* threads per CTA */
    uint32_t status;     /* raw device status word */
    uint64_t batches;    /* warp iterations that relaxed records */
    uint64_t idle;       /* warp iterations that found nothing to do */
} mlmq_solve_stats;
int mlmq_solver_stats(mlmq_solver *s, mlmq_solve_stats *st);
void mlmq_solver_destroy(mlmq_solver *s);

/* One-shot host-buffer call: upload the CSR, solve every source in srcs one
 * after another, copy each distance array to h_dist (nsrc x n, row-major).
 * This is the whole user-facing path with host buffers. */
int mlmq_solve_host(int n, int64_t m, const int *row, const int *col, const int *w,
                    int nsrc, const int *srcs, int *h_dist, const mlmq_config *cfg);

/* ---- 2c. batched multi-source solve ---------------------------------------
 * Many queries -- sources on one graph, or on several graphs of uneven size
 * -- in ONE persistent launch.  Replaces the reference's back-to-back solver
 * runs per source (SSSP/main.cu:213-307).  Each query slot owns a distance
 * array of max_vertices entries and its own queue rings; the CTAs of the
 * launch are split into one contiguous group per slot. */
typedef struct mlmq_batch mlmq_batch;
/* cfg may be NULL: mlmq_config_default() with 8 worker warps per CTA.
 * Per-slot rings default to 2^18 slots (L2) and 2^20 slots (L3). */
/* max_vertices bounds n + mlmq_graph_pieces() of every graph a launch uses. */
int mlmq_batch_create(int max_queries, int max_vertices, const mlmq_config *cfg,
                      mlmq_batch **out);
int mlmq_batch_info(const mlmq_batch *b, int *grid, int *block, int *max_queries);
/* Enqueues one launch solving query q from srcs[q] on graphs[q], q < nq.
 * use_graph != 0: the launch (parameter upload, kernel, status download) is
 * captured in a CUDA graph the first time a query set is seen and replayed
 * while the set is unchanged.  A run while the previous launch is
 * outstanding waits for it first (the query table and workspace are
 * shared); the earlier outcome is then not reported. */
int mlmq_batch_run(mlmq_batch *b, int nq, const mlmq_graph *const *graphs, const int *srcs,
                   int use_graph, void *stream);
/* Blocks until the launch ends; the first failing query's MLMQ_ERR_* code. */
int mlmq_batch_wait(mlmq_batch *b);
int mlmq_batch_query_status(const mlmq_batch *b, int q, unsigned *status,
                            mlmq_solve_stats *st);
int mlmq_batch_dist(mlmq_batch *b, int q, int **d_dist);
int mlmq_batch_copy_dist(mlmq_batch *b, int q, int *h_dist);
/* Copies the first `count` 32-bit words of query q's queue control block as
 * they were when its last launch ended (queue counters, `first`, status; the
 * layout is device_common.cuh's ctl namespace): a snapshot for diagnosing a
 * solve that timed out, the role of the reference's hang-diagnostic counters
 * (SSSP/sssp_run.cu HANG_DIAG, L3_LIVE_SNAPSHOT). */
int mlmq_batch_control(const mlmq_batch *b, int q, unsigned *words, int count);
void mlmq_batch_destroy(mlmq_batch *b);

/* ---- 2d. continuous-batching server ---------------------------------------
 * No counterpart in the reference (its only multi-query form is the
 * back-to-back batch above).  One persistent launch serves single-source
 * queries on HBM-resident device graphs as they arrive: the grid is split
 * into `slots` CTA groups; a submitted query goes to a free slot, its work
 * overlaps the other slots' queries on the device, and its distances are
 * copied to the caller's host buffer when it finishes.  Slots are admitted
 * by free device memory: at creation the server takes as many of the
 * requested slots as fit in free memory minus a 2 GiB reserve.  The launch
 * ends after lifetime_ms or mlmq_server_stop. */
typedef struct mlmq_server mlmq_server;
int mlmq_server_create(int slots, int max_vertices, const mlmq_config *cfg, int lifetime_ms,
                       mlmq_server **out);
/* As mlmq_server_create with slots of different sizes: slot s gets
 * slot_ctas[s] CTAs (their sum must fit the GPU's co-resident grid).  A
 * query asks for a slot size with mlmq_server_submit_cfg's knobs->work_blocks
 * and gets the smallest free slot of at least that many CTAs: small slots
 * suit latency-bound queries (many run side by side), wide ones
 * throughput-bound queries.  MLMQ_ERR_NOMEM if the slots do not all fit in
 * device memory. */
int mlmq_server_create_layout(int slots, const int *slot_ctas, int max_vertices,
                              const mlmq_config *cfg, int lifetime_ms, mlmq_server **out);
/* CTAs of each slot (up to `max` entries); *count = number of slots. */
int mlmq_server_layout(const mlmq_server *sv, int *slot_ctas, int max, int *count);
int mlmq_server_info(const mlmq_server *sv, int *slots, int *grid, int *block);
/* Non-blocking.  MLMQ_ERR_BUSY when every slot is taken; h_out (n ints) must
 * stay valid until the ticket is reported by mlmq_server_poll. */
int mlmq_server_submit(mlmq_server *sv, const mlmq_graph *g, int src, int *h_out,
                       uint64_t *ticket);
/* As mlmq_server_submit, with this query's delta, topup, l1_ahead,
 * bucket_max and bucket_sync taken from *knobs, and knobs->work_blocks = the smallest slot
 * (CTAs) it may run in (the other fields are fixed per server and ignored;
 * NULL = the server's configuration, any slot), so queries on graphs of
 * different shapes can each run their own tuned settings in one server. */
int mlmq_server_submit_cfg(mlmq_server *sv, const mlmq_graph *g, int src,
                           const mlmq_config *knobs, int *h_out, uint64_t *ticket);
/* Advances finished queries (result copy-out) and reports up to `max`
 * completed tickets with their MLMQ_ERR_* status. */
int mlmq_server_poll(mlmq_server *sv, uint64_t *tickets, int *statuses, int max, int *count);
/* As mlmq_server_poll, with each query's device time in ns from its slot
 * taking the command to the slot reporting the result (the solve without
 * host-side queueing and result copy-out); solve_ns may be NULL. */
int mlmq_server_poll_timed(mlmq_server *sv, uint64_t *tickets, int *statuses,
                           uint64_t *solve_ns, int max, int *count);
/* One finished served query. */
typedef struct mlmq_served_result {
    uint64_t ticket;
    int status;        /* MLMQ_ERR_* */
    uint64_t solve_ns; /* device time, as mlmq_server_poll_timed */
    uint64_t digest;   /* fingerprint of the distances the slot produced,
                          computed on the device (mlmq_dist_digest's
                          definition); 0 when the query failed */
} mlmq_served_result;
/* As mlmq_server_poll_timed, with each query's result digest: a caller can
 * check every served result against a reference digest without keeping the
 * distance arrays. */
int mlmq_server_poll_results(mlmq_server *sv, mlmq_served_result *out, int max, int *count);
/* Digest of a host distance array: the sum, modulo 2^64, of
 * mix64((v << 32) | (uint32_t)dist[v]) over v < n, mix64 being the
 * SplitMix64 output function.  Equal arrays give equal digests; a sum of
 * per-vertex terms, so the device computes it in any order. */
uint64_t mlmq_dist_digest(const int *dist, int64_t n);
/* Slots that are busy or out of service; MLMQ_ERR_STATE once the server
 * kernel has ended. */
int mlmq_server_busy_slots(mlmq_server *sv, int *busy);
int mlmq_server_stop(mlmq_server *sv);
void mlmq_server_destroy(mlmq_server *sv);

/* ---- 2e. single-source solve that allocates nothing ----------------------
 * No counterpart in the reference: the reference solver allocates its queue
 * storage with cudaMalloc on every run (sssp_run.cu:777-778).
 *
 * For callers that must not allocate device memory while they solve: code
 * whose device memory is owned by a framework's pool allocator, a process
 * that reserved all device memory up front, or a real-time path where an
 * allocation could block or fail.  The queue workspace is a fixed array in
 * the library's device image (MLMQ_NOALLOC_WORKSPACE_BYTES, about 26 MiB),
 * held on each device from the time the library's device code is loaded
 * there (at the latest, the first call) until the process exits.  The
 * caller passes the device CSR (d_row[n+1], d_col[m], d_w[m], read in
 * place) and the output d_dist[n]; nothing else is allocated.
 *
 *  - Graphs above MLMQ_NOALLOC_MAX_VERTICES vertices or MLMQ_NOALLOC_MAX_ARCS
 *    arcs, and bucket_num > 16, return MLMQ_ERR_RANGE before any work; at
 *    most 8 worker warps per CTA are used.
 *  - cfg may be NULL (mlmq_config_default).  The call runs on `stream`
 *    (a cudaStream_t, NULL = legacy default stream) and returns when the
 *    solve has finished, with its status.
 *  - The first call on a device looks up the workspace address and clears
 *    it; make that first call before any stream capture on that device.
 *    The set-up belongs to the device's CUDA context: after a
 *    cudaDeviceReset the next call repeats it.
 *  - All calls share the one workspace and it keeps the last call's
 *    contents: calls whose kernels overlap on the GPU (two host threads,
 *    two streams) race and corrupt each other's results.  Serialise them. */
#define MLMQ_NOALLOC_MAX_VERTICES (1 << 20)
#define MLMQ_NOALLOC_MAX_ARCS (1 << 20)
#define MLMQ_NOALLOC_WORKSPACE_BYTES 26346816
int mlmq_sssp_solve_noalloc(int n, int m, const int *d_row, const int *d_col, const int *d_w,
                            int src, int *d_dist, const mlmq_config *cfg, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* MLMQ_B200_H */
