/*
 * oracle/workload.c -- the benchmark's synthetic graphs, restated in plain C
 * for the reference arm of bench.py.
 *
 * TEST INFRASTRUCTURE ONLY.  bench.py --impl reference times the reference's
 * own CPU solver on the same graph the GPU arm solves; it must not load the
 * product library to build that graph.  These functions restate the
 * product's seeded generators (mlmq_hgraph_grid, mlmq_hgraph_knn,
 * mlmq_hgraph_rmat) and produce the same CSR byte for byte;
 * tests/test_oracle.py compares the two, and bench.py prints a digest of
 * the graph in both arms' configs.
 *
 * Every random draw is counter-based: SplitMix64's output function (Steele,
 * Lea and Flood, 2014) of (seed, stream, index), so the graph depends only
 * on the arguments.  Arrays are malloc()ed; oracle_free releases them.
 */
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define W_OK 0
#define W_ERR_ARG (-2)
#define W_ERR_NOMEM (-6)
#define W_ERR_RANGE (-8)

static uint64_t mix(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
static uint64_t draw(uint64_t seed, uint64_t stream, uint64_t idx) {
    return mix(mix(seed ^ (stream * 0xD1B54A32D192ED03ull)) ^ idx);
}
static double to_unit(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }
static int to_range(uint64_t h, int lo, int hi) {
    uint64_t span = (uint64_t)((int64_t)hi - (int64_t)lo + 1);
    return (int)((int64_t)lo + (int64_t)(((h >> 32) * span) >> 32));
}

void oracle_free(void *p) { free(p); }

/* ---- CSR output ---------------------------------------------------------- */
typedef struct {
    int n;
    long long m;
    int *row, *col, *w;
} csr;

static int cmp_arc(const void *a, const void *b) {
    const int *x = (const int *)a, *y = (const int *)b;
    if (x[0] != y[0]) return x[0] < y[0] ? -1 : 1;
    return x[1] < y[1] ? -1 : (x[1] > y[1]);
}

/* Orders each row's arcs by (destination, weight). */
static int sort_each_row(csr *g) {
    int maxd = 0;
    for (int u = 0; u < g->n; u++)
        if (g->row[u + 1] - g->row[u] > maxd) maxd = g->row[u + 1] - g->row[u];
    int *tmp = (int *)malloc(sizeof(int) * 2 * (size_t)(maxd ? maxd : 1));
    if (!tmp) return W_ERR_NOMEM;
    for (int u = 0; u < g->n; u++) {
        int b = g->row[u], d = g->row[u + 1] - b;
        if (d < 2) continue;
        for (int i = 0; i < d; i++) {
            tmp[2 * i] = g->col[b + i];
            tmp[2 * i + 1] = g->w[b + i];
        }
        qsort(tmp, (size_t)d, 2 * sizeof(int), cmp_arc);
        for (int i = 0; i < d; i++) {
            g->col[b + i] = tmp[2 * i];
            g->w[b + i] = tmp[2 * i + 1];
        }
    }
    free(tmp);
    return W_OK;
}

static void csr_release(csr *g) {
    free(g->row);
    free(g->col);
    free(g->w);
    g->row = g->col = g->w = NULL;
}

static int hand_out(csr *g, int *n, long long *m, int **row, int **col, int **w) {
    *n = g->n;
    *m = g->m;
    *row = g->row;
    *col = g->col;
    *w = g->w;
    return W_OK;
}

/* ---- road-like grid (mlmq_hgraph_grid) ------------------------------------
 * Undirected edge ids: 2v for (v, v+1), 2v+1 for (v, v+width); an edge is
 * kept when its uniform draw (stream 1) is >= drop_p; both arcs carry one
 * weight (stream 2).  Each row lists up, left, right, down. */
int oracle_gen_grid(int width, int height, double drop_p, int wmin, int wmax, uint64_t seed,
                    int *n_out, long long *m_out, int **row, int **col, int **w) {
    if (width <= 0 || height <= 0 || wmin < 0 || wmax < wmin || drop_p < 0 || drop_p > 1)
        return W_ERR_ARG;
    long long n64 = (long long)width * height;
    if (n64 >= INT_MAX) return W_ERR_RANGE;
    csr g = {(int)n64, 0, NULL, NULL, NULL};
    g.row = (int *)calloc((size_t)g.n + 1, sizeof(int));
    if (!g.row) return W_ERR_NOMEM;
#define KEEP(e) (to_unit(draw(seed, 1, (uint64_t)(e))) >= drop_p)
#define WGT(e) to_range(draw(seed, 2, (uint64_t)(e)), wmin, wmax)
    for (int pass = 0; pass < 2; pass++) {
        for (long long v = 0; v < g.n; v++) {
            int x = (int)(v % width), y = (int)(v / width);
            int p = pass ? g.row[v] : 0, d = 0;
            long long ids[4], to[4];
            int k = 0;
            if (y > 0) { ids[k] = 2 * (v - width) + 1; to[k++] = v - width; }
            if (x > 0) { ids[k] = 2 * (v - 1); to[k++] = v - 1; }
            if (x + 1 < width) { ids[k] = 2 * v; to[k++] = v + 1; }
            if (y + 1 < height) { ids[k] = 2 * v + 1; to[k++] = v + width; }
            for (int i = 0; i < k; i++) {
                if (!KEEP(ids[i])) continue;
                if (pass) {
                    g.col[p] = (int)to[i];
                    g.w[p++] = WGT(ids[i]);
                } else {
                    d++;
                }
            }
            if (!pass) g.row[v + 1] = d;
        }
        if (!pass) {
            for (int i = 0; i < g.n; i++) g.row[i + 1] += g.row[i];
            g.m = g.row[g.n];
            g.col = (int *)malloc(sizeof(int) * (size_t)(g.m ? g.m : 1));
            g.w = (int *)malloc(sizeof(int) * (size_t)(g.m ? g.m : 1));
            if (!g.col || !g.w) {
                csr_release(&g);
                return W_ERR_NOMEM;
            }
        }
    }
#undef KEEP
#undef WGT
    return hand_out(&g, n_out, m_out, row, col, w);
}

/* ---- planar kNN (mlmq_hgraph_knn) -----------------------------------------
 * Points uniform in the unit square (streams 1, 2); ids follow the Morton
 * order of a G x G cell grid (G = floor(sqrt(n/2)), ties by point index);
 * each point's k nearest others by (squared distance, id), searched ring by
 * ring of cells until the k-th is no farther than the ring's inner edge;
 * pairs symmetrised and deduplicated; weight = llround(scale * d) + 1. */
static uint32_t spread16(uint32_t x) {
    x &= 0xffff;
    x = (x | (x << 8)) & 0x00FF00FF;
    x = (x | (x << 4)) & 0x0F0F0F0F;
    x = (x | (x << 2)) & 0x33333333;
    x = (x | (x << 1)) & 0x55555555;
    return x;
}

static int cmp_u64(const void *a, const void *b) {
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return x < y ? -1 : (x > y);
}

typedef struct {
    double d;
    int u;
} cand;

/* (d, u) < (e, v) lexicographically. */
static int cand_less(double d, int u, const cand *c) { return d < c->d || (d == c->d && u < c->u); }

int oracle_gen_knn(int npoints, int k, double scale, uint64_t seed, int *n_out, long long *m_out,
                   int **row, int **col, int **w) {
    if (npoints < 2 || k < 1 || k >= npoints || k > 16 || !(scale > 0)) return W_ERR_ARG;
    const int n = npoints;
    int rc = W_OK;
    double *px = (double *)malloc(sizeof(double) * (size_t)n);
    double *py = (double *)malloc(sizeof(double) * (size_t)n);
    double *x = (double *)malloc(sizeof(double) * (size_t)n);
    double *y = (double *)malloc(sizeof(double) * (size_t)n);
    uint64_t *key = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)n);
    int *nbr = (int *)malloc(sizeof(int) * (size_t)n * (size_t)k);
    int G = (int)sqrt(n / 2.0);
    if (G < 1) G = 1;
    if (G > 65535) G = 65535;
    int *cbeg = (int *)calloc((size_t)G * G, sizeof(int));
    int *cend = (int *)calloc((size_t)G * G, sizeof(int));
    uint64_t *pairs = NULL;
    csr g = {n, 0, NULL, NULL, NULL};
    if (!px || !py || !x || !y || !key || !nbr || !cbeg || !cend) {
        rc = W_ERR_NOMEM;
        goto done;
    }
#define CELL(v) ((int)((v) * G) < G - 1 ? (int)((v) * G) : G - 1)
    for (int i = 0; i < n; i++) {
        px[i] = to_unit(draw(seed, 1, (uint64_t)i));
        py[i] = to_unit(draw(seed, 2, (uint64_t)i));
        uint32_t cx = (uint32_t)CELL(px[i]), cy = (uint32_t)CELL(py[i]);
        key[i] = ((uint64_t)(spread16(cx) | (spread16(cy) << 1)) << 32) | (uint32_t)i;
    }
    qsort(key, (size_t)n, sizeof(uint64_t), cmp_u64);
    for (int v = 0; v < n; v++) {
        int i = (int)(key[v] & 0xffffffffu);
        x[v] = px[i];
        y[v] = py[i];
    }
    for (int v = 0; v < n; v++) {
        size_t c = (size_t)CELL(y[v]) * G + CELL(x[v]);
        if (cend[c] == 0) cbeg[c] = v;
        cend[c] = v + 1;
    }
    {
        const double cs = 1.0 / G;
        cand best[17];
        for (int v = 0; v < n; v++) {
            int have = 0;
            const int cx = CELL(x[v]), cy = CELL(y[v]);
            for (int r = 0;; r++) {
                for (int yy = cy - r; yy <= cy + r; yy++) {
                    if (yy < 0 || yy >= G) continue;
                    const int full = (yy == cy - r || yy == cy + r);
                    for (int xx = cx - r; xx <= cx + r; xx += (full ? 1 : 2 * r)) {
                        if (xx >= 0 && xx < G) {
                            size_t c = (size_t)yy * G + xx;
                            for (int u = cbeg[c]; u < cend[c]; u++) {
                                if (u == v) continue;
                                double dx = x[u] - x[v], dy = y[u] - y[v];
                                double d = dx * dx + dy * dy;
                                /* keep the k smallest (d, u), sorted */
                                if (have == k && !cand_less(d, u, &best[k - 1])) continue;
                                int p = have < k ? have++ : k - 1;
                                while (p > 0 && cand_less(d, u, &best[p - 1])) {
                                    best[p] = best[p - 1];
                                    p--;
                                }
                                best[p].d = d;
                                best[p].u = u;
                            }
                        }
                        if (r == 0) break;
                    }
                }
                if (have >= k) {
                    double lim = r * cs;
                    if (best[k - 1].d <= lim * lim) break;
                }
                if (r > 2 * G) break;
            }
            for (int j = 0; j < k; j++) nbr[(size_t)v * k + j] = best[j].u;
        }
    }
#undef CELL
    pairs = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)n * (size_t)k);
    if (!pairs) {
        rc = W_ERR_NOMEM;
        goto done;
    }
    size_t np = 0;
    for (int v = 0; v < n; v++)
        for (int j = 0; j < k; j++) {
            int u = nbr[(size_t)v * k + j];
            int a = u < v ? u : v, c = u < v ? v : u;
            pairs[np++] = ((uint64_t)a << 32) | (uint32_t)c;
        }
    qsort(pairs, np, sizeof(uint64_t), cmp_u64);
    size_t uniq = 0;
    for (size_t i = 0; i < np; i++)
        if (uniq == 0 || pairs[i] != pairs[uniq - 1]) pairs[uniq++] = pairs[i];
    if (2 * (long long)uniq >= INT_MAX) {
        rc = W_ERR_RANGE;
        goto done;
    }
    g.m = 2 * (long long)uniq;
    g.row = (int *)calloc((size_t)n + 1, sizeof(int));
    g.col = (int *)malloc(sizeof(int) * (size_t)g.m);
    g.w = (int *)malloc(sizeof(int) * (size_t)g.m);
    int *fill = (int *)malloc(sizeof(int) * (size_t)n);
    if (!g.row || !g.col || !g.w || !fill) {
        free(fill);
        csr_release(&g);
        rc = W_ERR_NOMEM;
        goto done;
    }
    for (size_t i = 0; i < uniq; i++) {
        g.row[(pairs[i] >> 32) + 1]++;
        g.row[(pairs[i] & 0xffffffffu) + 1]++;
    }
    for (int i = 0; i < n; i++) g.row[i + 1] += g.row[i];
    memcpy(fill, g.row, sizeof(int) * (size_t)n);
    for (size_t i = 0; i < uniq; i++) {
        int a = (int)(pairs[i] >> 32), c = (int)(pairs[i] & 0xffffffffu);
        double dx = x[a] - x[c], dy = y[a] - y[c];
        double wd = (double)llround(scale * sqrt(dx * dx + dy * dy)) + 1.0;
        if (wd >= INT_MAX) {
            free(fill);
            csr_release(&g);
            rc = W_ERR_RANGE;
            goto done;
        }
        g.col[fill[a]] = c;
        g.w[fill[a]++] = (int)wd;
        g.col[fill[c]] = a;
        g.w[fill[c]++] = (int)wd;
    }
    free(fill);
    rc = sort_each_row(&g);
    if (rc) csr_release(&g);
done:
    free(px);
    free(py);
    free(x);
    free(y);
    free(key);
    free(nbr);
    free(cbeg);
    free(cend);
    free(pairs);
    if (rc) return rc;
    return hand_out(&g, n_out, m_out, row, col, w);
}

/* ---- R-MAT (mlmq_hgraph_rmat) ---------------------------------------------
 * Sample i draws 16 bits per level from draw(seed, 3, 8i + level/4) (four
 * levels per draw) against the quadrant thresholds round(a, a+b, a+b+c x
 * 2^16); self-loops dropped; each source's targets sorted and deduplicated;
 * weight of (u, v) from draw(seed, 4, u << 32 | v). */
static int cmp_int(const void *a, const void *b) {
    int x = *(const int *)a, y = *(const int *)b;
    return x < y ? -1 : (x > y);
}

int oracle_gen_rmat(int scale, int edge_factor, double a, double b, double c, int wmin, int wmax,
                    uint64_t seed, int *n_out, long long *m_out, int **row, int **col, int **w) {
    if (scale < 1 || scale > 30 || edge_factor < 1 || a < 0 || b < 0 || c < 0 || a + b + c > 1 ||
        wmin < 0 || wmax < wmin)
        return W_ERR_ARG;
    long long n64 = 1ll << scale, samples = n64 * edge_factor;
    if (n64 >= INT_MAX || samples >= INT_MAX) return W_ERR_RANGE;
    const int n = (int)n64;
    const uint32_t ta = (uint32_t)llround(a * 65536.0);
    const uint32_t tb = (uint32_t)llround((a + b) * 65536.0);
    const uint32_t tc = (uint32_t)llround((a + b + c) * 65536.0);
    int *su = (int *)malloc(sizeof(int) * (size_t)samples);
    int *sv = (int *)malloc(sizeof(int) * (size_t)samples);
    int *deg = (int *)calloc((size_t)n + 1, sizeof(int));
    csr g = {n, 0, NULL, NULL, NULL};
    int *tmp = NULL, *cnt = NULL;
    int rc = W_OK;
    if (!su || !sv || !deg) {
        rc = W_ERR_NOMEM;
        goto done;
    }
    for (long long i = 0; i < samples; i++) {
        uint32_t u = 0, v = 0;
        uint64_t h = 0;
        for (int lvl = 0; lvl < scale; lvl++) {
            if ((lvl & 3) == 0) h = draw(seed, 3, (uint64_t)i * 8 + (uint64_t)(lvl >> 2));
            uint32_t r = (uint32_t)(h & 0xffff);
            h >>= 16;
            uint32_t bu = r >= tb, bv = (r >= ta && r < tb) || r >= tc;
            u = (u << 1) | bu;
            v = (v << 1) | bv;
        }
        su[i] = (int)u;
        sv[i] = (int)v;
        if (u != v) deg[u + 1]++;
    }
    for (int i = 0; i < n; i++) deg[i + 1] += deg[i];
    tmp = (int *)malloc(sizeof(int) * (size_t)(deg[n] ? deg[n] : 1));
    cnt = (int *)malloc(sizeof(int) * (size_t)n);
    if (!tmp || !cnt) {
        rc = W_ERR_NOMEM;
        goto done;
    }
    memcpy(cnt, deg, sizeof(int) * (size_t)n);
    for (long long i = 0; i < samples; i++)
        if (su[i] != sv[i]) tmp[cnt[su[i]]++] = sv[i];
    g.row = (int *)calloc((size_t)n + 1, sizeof(int));
    if (!g.row) {
        rc = W_ERR_NOMEM;
        goto done;
    }
    for (int u = 0; u < n; u++) {
        int bgn = deg[u], d = deg[u + 1] - bgn, keep = 0;
        qsort(tmp + bgn, (size_t)d, sizeof(int), cmp_int);
        for (int j = 0; j < d; j++)
            if (keep == 0 || tmp[bgn + j] != tmp[bgn + keep - 1]) tmp[bgn + keep++] = tmp[bgn + j];
        cnt[u] = keep;
        g.row[u + 1] = g.row[u] + keep;
    }
    g.m = g.row[n];
    g.col = (int *)malloc(sizeof(int) * (size_t)(g.m ? g.m : 1));
    g.w = (int *)malloc(sizeof(int) * (size_t)(g.m ? g.m : 1));
    if (!g.col || !g.w) {
        csr_release(&g);
        rc = W_ERR_NOMEM;
        goto done;
    }
    for (int u = 0; u < n; u++)
        for (int j = 0; j < cnt[u]; j++) {
            int v = tmp[deg[u] + j], p = g.row[u] + j;
            g.col[p] = v;
            g.w[p] = to_range(draw(seed, 4, ((uint64_t)u << 32) | (uint32_t)v), wmin, wmax);
        }
done:
    free(su);
    free(sv);
    free(deg);
    free(tmp);
    free(cnt);
    if (rc) return rc;
    return hand_out(&g, n_out, m_out, row, col, w);
}
