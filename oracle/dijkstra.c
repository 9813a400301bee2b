/*
 * oracle/dijkstra.c -- CPU oracle for the delta-stepping SSSP hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: tests/, the smoke
 * check in __graft_entry__.py and the cpu_baseline leg of bench.py load it.
 * The product (mlmq_tpds_withl3_b200 and libmlmq_b200.so) never links,
 * imports or calls it, and has no CPU fallback.
 *
 * It restates, in plain C, the two CPU shortest-path routines of the
 * reference project (hideoze/mlmq_tpds_withl3):
 *
 *   oracle_sssp_i32  follows evidence/l3_supplement_20260921_v2/single_source/
 *                    SSSP/main.cu:47-117 (sssp_sequential): lazy-deletion
 *                    Dijkstra over a binary min-heap of (dist, id), a done[]
 *                    mark per settled vertex, int32 distances initialised to
 *                    INT_MAX, and total_work = sum of out-degrees of settled
 *                    vertices (main.cu:71).
 *   oracle_sssp_i64  follows scripts/multigpu/supplement_graph.cpp:32-43: the
 *                    same search with 64-bit sums that refuses any finite
 *                    distance >= INT_MAX ("unrepresentable distance").
 *
 * Both write INT_MAX for unreachable vertices, as the reference does.
 * Shortest-path distances with non-negative integer weights are unique, so
 * the heap's tie order does not change any output.
 *
 * Where the reference's int32 routine would overflow (a sum >= 2^31, undefined
 * behaviour in C++), oracle_sssp_i32 returns ORACLE_ERR_OVERFLOW instead of
 * producing a value.
 *
 * Pinning: tests/golden/make_golden.py runs the reference's own
 * sssp_sequential, compiled from the reference sources by oracle/Makefile into
 * oracle/_ref/, on the committed fixtures; tests/test_oracle.py checks these
 * functions against those golden distances and work counts.
 */
#include <limits.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_OK 0
#define ORACLE_ERR_ARG (-2)
#define ORACLE_ERR_NOMEM (-6)
#define ORACLE_ERR_OVERFLOW (-8)

typedef struct {
    int64_t d;
    int32_t v;
} heap_item;

typedef struct {
    heap_item *a;
    size_t n, cap;
} heap;

static int heap_push(heap *h, int64_t d, int32_t v) {
    if (h->n == h->cap) {
        size_t nc = h->cap ? h->cap * 2 : 1024;
        heap_item *na = (heap_item *)realloc(h->a, nc * sizeof(heap_item));
        if (!na) return ORACLE_ERR_NOMEM;
        h->a = na;
        h->cap = nc;
    }
    size_t i = h->n++;
    while (i > 0) {
        size_t p = (i - 1) >> 1;
        if (h->a[p].d <= d) break;
        h->a[i] = h->a[p];
        i = p;
    }
    h->a[i].d = d;
    h->a[i].v = v;
    return ORACLE_OK;
}

static heap_item heap_pop(heap *h) {
    heap_item top = h->a[0];
    heap_item last = h->a[--h->n];
    size_t i = 0, n = h->n;
    for (;;) {
        size_t c = 2 * i + 1;
        if (c >= n) break;
        if (c + 1 < n && h->a[c + 1].d < h->a[c].d) c++;
        if (h->a[c].d >= last.d) break;
        h->a[i] = h->a[c];
        i = c;
    }
    if (n) h->a[i] = last;
    return top;
}

static int check_args(int n, const int *row, const int *col, const int *w, int src) {
    if (n <= 0 || !row || src < 0 || src >= n) return ORACLE_ERR_ARG;
    if (row[n] > 0 && (!col || !w)) return ORACLE_ERR_ARG;
    return ORACLE_OK;
}

/* SS/SSSP/main.cu:47-117.  dist[] is written in full (INT_MAX, then the
 * search); *total_work receives the reference's work count (arcs out of
 * settled vertices).  Sums are formed in 64 bits so that an int32 overflow is
 * reported rather than wrapped. */
int oracle_sssp_i32(int n, const int *row, const int *col, const int *w, int src,
                    int *dist, long long *total_work) {
    int rc = check_args(n, row, col, w, src);
    if (rc) return rc;
    unsigned char *done = (unsigned char *)calloc((size_t)n, 1);
    if (!done) return ORACLE_ERR_NOMEM;
    heap h = {0, 0, 0};
    for (int i = 0; i < n; i++) dist[i] = INT_MAX;
    dist[src] = 0;
    long long work = 0;
    rc = heap_push(&h, 0, src);
    while (rc == ORACLE_OK && h.n) {
        heap_item it = heap_pop(&h);
        int u = it.v;
        if (done[u]) continue;
        done[u] = 1;
        work += row[u + 1] - row[u];
        int64_t du = dist[u];
        for (int e = row[u]; e < row[u + 1]; e++) {
            int v = col[e];
            int64_t nd = du + (int64_t)w[e];
            if (nd > INT_MAX) {
                /* main.cu:78 forms this sum in int: it would overflow here. */
                rc = ORACLE_ERR_OVERFLOW;
                break;
            }
            if ((int64_t)dist[v] > nd) {
                dist[v] = (int)nd;
                rc = heap_push(&h, nd, v);
                if (rc) break;
            }
        }
    }
    free(h.a);
    free(done);
    if (total_work) *total_work = work;
    return rc;
}

/* scripts/multigpu/supplement_graph.cpp:32-43: 64-bit distances; an entry is
 * stale when its key differs from the current distance; a finite distance
 * >= INT_MAX is an error.  *reached and *max_dist mirror the routine's
 * "ORACLE ... reached= max_distance=" report. */
int oracle_sssp_i64(int n, const int *row, const int *col, const int *w, int src,
                    int *dist, int *reached, long long *max_dist) {
    int rc = check_args(n, row, col, w, src);
    if (rc) return rc;
    const int64_t INF = (int64_t)1 << 62;
    int64_t *d = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
    if (!d) return ORACLE_ERR_NOMEM;
    for (int i = 0; i < n; i++) d[i] = INF;
    d[src] = 0;
    heap h = {0, 0, 0};
    rc = heap_push(&h, 0, src);
    while (rc == ORACLE_OK && h.n) {
        heap_item it = heap_pop(&h);
        int u = it.v;
        if (it.d != d[u]) continue;
        for (int e = row[u]; e < row[u + 1]; e++) {
            int v = col[e];
            int64_t nd = it.d + (int64_t)w[e];
            if (nd < d[v]) {
                d[v] = nd;
                rc = heap_push(&h, nd, v);
                if (rc) break;
            }
        }
    }
    free(h.a);
    int cnt = 0;
    int64_t mx = 0;
    for (int i = 0; i < n && rc == ORACLE_OK; i++) {
        if (d[i] == INF) {
            dist[i] = INT_MAX;
            continue;
        }
        if (d[i] >= INT_MAX) {
            rc = ORACLE_ERR_OVERFLOW;
            break;
        }
        dist[i] = (int)d[i];
        cnt++;
        if (d[i] > mx) mx = d[i];
    }
    free(d);
    if (reached) *reached = cnt;
    if (max_dist) *max_dist = mx;
    return rc;
}

/* Many independent sources over a thread pool: the reference's multi-source
 * form runs one full solve per source (SSSP/main.cu:396-433).  dist is
 * nsrc x n, row-major by source; work (optional) is nsrc entries. */
typedef struct {
    int n;
    const int *row, *col, *w;
    int nsrc;
    const int *srcs;
    int *dist;
    long long *work;
    int next;
    int rc;
    pthread_mutex_t mu;
} many_job;

static void *many_worker(void *arg) {
    many_job *j = (many_job *)arg;
    for (;;) {
        pthread_mutex_lock(&j->mu);
        int k = j->next++;
        pthread_mutex_unlock(&j->mu);
        if (k >= j->nsrc) break;
        long long wk = 0;
        int rc = oracle_sssp_i32(j->n, j->row, j->col, j->w, j->srcs[k],
                                 j->dist + (size_t)k * (size_t)j->n, &wk);
        if (j->work) j->work[k] = wk;
        if (rc) {
            pthread_mutex_lock(&j->mu);
            if (!j->rc) j->rc = rc;
            pthread_mutex_unlock(&j->mu);
        }
    }
    return NULL;
}

int oracle_sssp_many(int n, const int *row, const int *col, const int *w, int nsrc,
                     const int *srcs, int *dist, long long *work, int nthreads) {
    if (nsrc < 0 || (nsrc && (!srcs || !dist))) return ORACLE_ERR_ARG;
    if (nthreads < 1) nthreads = 1;
    if (nthreads > nsrc) nthreads = nsrc ? nsrc : 1;
    many_job j;
    j.n = n; j.row = row; j.col = col; j.w = w;
    j.nsrc = nsrc; j.srcs = srcs; j.dist = dist; j.work = work;
    j.next = 0; j.rc = 0;
    pthread_mutex_init(&j.mu, NULL);
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nthreads);
    if (!th) return ORACLE_ERR_NOMEM;
    int started = 0;
    for (int t = 0; t < nthreads; t++)
        if (pthread_create(&th[t], NULL, many_worker, &j) == 0) started++;
        else break;
    if (!started) many_worker(&j);
    for (int t = 0; t < started; t++) pthread_join(th[t], NULL);
    free(th);
    pthread_mutex_destroy(&j.mu);
    return j.rc;
}

/* Fingerprint of a distance array, for checking results that are not kept
 * in full (served queries): the sum, modulo 2^64, of
 * splitmix64_out((v << 32) | (uint32)dist[v]) over every vertex v, where
 * splitmix64_out is the output function of SplitMix64 (Steele, Lea and
 * Flood, 2014).  The library computes the same sum on the device
 * (mlmq_dist_digest defines it for callers); two arrays with equal digests
 * are equal except with probability about 2^-64 per comparison. */
static uint64_t splitmix64_out(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

uint64_t oracle_digest(int n, const int *dist) {
    uint64_t s = 0;
    for (int v = 0; v < n; v++) s += splitmix64_out(((uint64_t)(uint32_t)v << 32) | (uint32_t)dist[v]);
    return s;
}

/* Many sources, keeping only each result's digest, total_work and reached
 * count (memory: one distance array per thread). */
typedef struct {
    int n;
    const int *row, *col, *w;
    int nsrc;
    const int *srcs;
    uint64_t *digest;
    long long *work;
    int *reached;
    int next;
    int rc;
    pthread_mutex_t mu;
} digest_job;

static void *digest_worker(void *arg) {
    digest_job *j = (digest_job *)arg;
    int *d = (int *)malloc(sizeof(int) * (size_t)j->n);
    for (;;) {
        pthread_mutex_lock(&j->mu);
        int k = j->next++;
        if (!d && !j->rc) j->rc = ORACLE_ERR_NOMEM;
        pthread_mutex_unlock(&j->mu);
        if (k >= j->nsrc || !d) break;
        long long wk = 0;
        int rc = oracle_sssp_i32(j->n, j->row, j->col, j->w, j->srcs[k], d, &wk);
        j->digest[k] = oracle_digest(j->n, d);
        if (j->work) j->work[k] = wk;
        if (j->reached) {
            int c = 0;
            for (int v = 0; v < j->n; v++) c += d[v] != INT_MAX;
            j->reached[k] = c;
        }
        if (rc) {
            pthread_mutex_lock(&j->mu);
            if (!j->rc) j->rc = rc;
            pthread_mutex_unlock(&j->mu);
        }
    }
    free(d);
    return NULL;
}

int oracle_sssp_digest_many(int n, const int *row, const int *col, const int *w, int nsrc,
                            const int *srcs, uint64_t *digest, long long *work, int *reached,
                            int nthreads) {
    if (nsrc < 0 || (nsrc && (!srcs || !digest))) return ORACLE_ERR_ARG;
    if (nthreads < 1) nthreads = 1;
    if (nthreads > nsrc) nthreads = nsrc ? nsrc : 1;
    digest_job j;
    j.n = n; j.row = row; j.col = col; j.w = w;
    j.nsrc = nsrc; j.srcs = srcs; j.digest = digest; j.work = work; j.reached = reached;
    j.next = 0; j.rc = 0;
    pthread_mutex_init(&j.mu, NULL);
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nthreads);
    if (!th) return ORACLE_ERR_NOMEM;
    int started = 0;
    for (int t = 0; t < nthreads; t++)
        if (pthread_create(&th[t], NULL, digest_worker, &j) == 0) started++;
        else break;
    if (!started) digest_worker(&j);
    for (int t = 0; t < started; t++) pthread_join(th[t], NULL);
    free(th);
    pthread_mutex_destroy(&j.mu);
    return j.rc;
}
