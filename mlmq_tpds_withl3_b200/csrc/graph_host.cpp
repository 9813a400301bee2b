// graph_host.cpp -- host-side graph layer of libmlmq_b200.so: seeded synthetic
// generators for the road-like grid, kNN and R-MAT workloads, the .gr v1
// binary CSR reader/writer, and CSR validation.
//
// .gr v1 layout (reference SSSP/csr_graph.cu:185-300 reader, :302-418 writer;
// validation rules of scripts/multigpu/supplement_graph.cpp:15-28):
//   u64 version=1, u64 edge_size=4, u64 n, u64 m,
//   u64 row_end[n], u32 dst[m], (u32 pad if m is odd), i32 weight[m],
// all little-endian.  The format must match byte for byte so that graphs move
// freely between the reference's tools and this library.
//
// Every generator is counter-based (splitmix64 of (seed, stream, index)), so
// the output depends only on its arguments, not on the thread count.
#include "mlmq_b200.h"

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <thread>
#include <vector>

#include "host_graph.h"

namespace {

inline uint64_t mix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
inline uint64_t hash3(uint64_t seed, uint64_t stream, uint64_t idx) {
    return mix64(mix64(seed ^ (stream * 0xD1B54A32D192ED03ull)) ^ idx);
}
inline double unit01(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }
// Uniform integer in [lo, hi] by multiply-shift of the top 32 bits.
inline int uniform_int(uint64_t h, int lo, int hi) {
    uint64_t range = (uint64_t)((int64_t)hi - (int64_t)lo + 1);
    return (int)((int64_t)lo + (int64_t)(((h >> 32) * range) >> 32));
}

int num_threads() {
    unsigned t = std::thread::hardware_concurrency();
    return t ? (int)std::min(t, 64u) : 4;
}

template <class F>
void parallel_for(int64_t n, F f) {
    int nt = num_threads();
    if (n < 65536 || nt <= 1) {
        f((int64_t)0, n, 0);
        return;
    }
    std::vector<std::thread> th;
    int64_t chunk = (n + nt - 1) / nt;
    for (int t = 0; t < nt; t++) {
        int64_t b = t * chunk, e = std::min(n, b + chunk);
        if (b >= e) break;
        th.emplace_back([=, &f] { f(b, e, t); });
    }
    for (auto &x : th) x.join();
}

// Validation of supplement_graph.cpp:26-28: monotone rows ending at m,
// destinations in range, non-negative weights.
int validate_csr(int n, int64_t m, const int *row, const int *col, const int *w) {
    if (n <= 0 || m < 0 || m >= INT_MAX || !row) return MLMQ_ERR_ARG;
    if (m > 0 && (!col || !w)) return MLMQ_ERR_ARG;
    if (row[0] != 0 || row[n] != m) return MLMQ_ERR_ARG;
    for (int u = 0; u < n; u++)
        if (row[u + 1] < row[u]) return MLMQ_ERR_ARG;
    std::atomic<int> bad(0);
    parallel_for(m, [&](int64_t b, int64_t e, int) {
        for (int64_t i = b; i < e; i++)
            if (col[i] < 0 || col[i] >= n || w[i] < 0) {
                bad.store(1);
                return;
            }
    });
    return bad.load() ? MLMQ_ERR_ARG : MLMQ_OK;
}

// Sorts each row's arcs by destination (weights follow), the canonical order
// used by every generator here.
void sort_rows(mlmq_host_graph &g) {
    parallel_for(g.n, [&](int64_t b, int64_t e, int) {
        std::vector<std::pair<int, int>> tmp;
        for (int64_t u = b; u < e; u++) {
            int rb = g.row[u], re = g.row[u + 1];
            if (re - rb < 2) continue;
            tmp.clear();
            for (int i = rb; i < re; i++) tmp.emplace_back(g.col[i], g.w[i]);
            std::sort(tmp.begin(), tmp.end());
            for (int i = rb; i < re; i++) {
                g.col[i] = tmp[i - rb].first;
                g.w[i] = tmp[i - rb].second;
            }
        }
    });
}

// Builds a symmetric CSR from unique undirected pairs (a < b) with weights.
int csr_from_pairs(int n, const std::vector<uint64_t> &pairs, const std::vector<int> &pw,
                   mlmq_host_graph &g) {
    int64_t m = 2 * (int64_t)pairs.size();
    if (m >= INT_MAX) return MLMQ_ERR_RANGE;
    g.n = n;
    g.m = m;
    g.row.assign((size_t)n + 1, 0);
    for (uint64_t p : pairs) {
        g.row[(p >> 32) + 1]++;
        g.row[(p & 0xffffffffu) + 1]++;
    }
    for (int i = 0; i < n; i++) g.row[i + 1] += g.row[i];
    g.col.resize((size_t)m);
    g.w.resize((size_t)m);
    std::vector<int> fill(g.row.begin(), g.row.end() - 1);
    for (size_t i = 0; i < pairs.size(); i++) {
        int a = (int)(pairs[i] >> 32), b = (int)(pairs[i] & 0xffffffffu);
        g.col[fill[a]] = b;
        g.w[fill[a]++] = pw[i];
        g.col[fill[b]] = a;
        g.w[fill[b]++] = pw[i];
    }
    sort_rows(g);
    return MLMQ_OK;
}

uint32_t morton16(uint32_t x) {
    x &= 0xffff;
    x = (x | (x << 8)) & 0x00FF00FF;
    x = (x | (x << 4)) & 0x0F0F0F0F;
    x = (x | (x << 2)) & 0x33333333;
    x = (x | (x << 1)) & 0x55555555;
    return x;
}

}  // namespace

extern "C" {

int mlmq_hgraph_grid(int width, int height, double drop_p, int wmin, int wmax, uint64_t seed,
                     mlmq_host_graph **out) {
    if (!out || width <= 0 || height <= 0 || wmin < 0 || wmax < wmin || drop_p < 0 ||
        drop_p > 1)
        return MLMQ_ERR_ARG;
    int64_t n64 = (int64_t)width * height;
    if (n64 >= INT_MAX) return MLMQ_ERR_RANGE;
    int n = (int)n64;
    auto *g = new (std::nothrow) mlmq_host_graph;
    if (!g) return MLMQ_ERR_NOMEM;
    // Undirected edge ids: 2*v for (v, v+1), 2*v+1 for (v, v+width).
    auto keep = [&](int64_t eid) { return unit01(hash3(seed, 1, (uint64_t)eid)) >= drop_p; };
    auto wgt = [&](int64_t eid) { return uniform_int(hash3(seed, 2, (uint64_t)eid), wmin, wmax); };
    try {
        g->n = n;
        g->row.assign((size_t)n + 1, 0);
        parallel_for(n, [&](int64_t b, int64_t e, int) {
            for (int64_t v = b; v < e; v++) {
                int x = (int)(v % width), y = (int)(v / width), d = 0;
                if (y > 0 && keep(2 * (v - width) + 1)) d++;
                if (x > 0 && keep(2 * (v - 1))) d++;
                if (x + 1 < width && keep(2 * v)) d++;
                if (y + 1 < height && keep(2 * v + 1)) d++;
                g->row[v + 1] = d;
            }
        });
        for (int i = 0; i < n; i++) g->row[i + 1] += g->row[i];
        g->m = g->row[n];
        g->col.resize((size_t)g->m);
        g->w.resize((size_t)g->m);
        parallel_for(n, [&](int64_t b, int64_t e, int) {
            for (int64_t v = b; v < e; v++) {
                int x = (int)(v % width), y = (int)(v / width);
                int p = g->row[v];
                // Destinations in increasing order: up, left, right, down.
                if (y > 0 && keep(2 * (v - width) + 1)) {
                    g->col[p] = (int)(v - width);
                    g->w[p++] = wgt(2 * (v - width) + 1);
                }
                if (x > 0 && keep(2 * (v - 1))) {
                    g->col[p] = (int)(v - 1);
                    g->w[p++] = wgt(2 * (v - 1));
                }
                if (x + 1 < width && keep(2 * v)) {
                    g->col[p] = (int)(v + 1);
                    g->w[p++] = wgt(2 * v);
                }
                if (y + 1 < height && keep(2 * v + 1)) {
                    g->col[p] = (int)(v + width);
                    g->w[p++] = wgt(2 * v + 1);
                }
            }
        });
    } catch (...) {
        delete g;
        return MLMQ_ERR_NOMEM;
    }
    *out = g;
    return MLMQ_OK;
}

int mlmq_hgraph_knn(int npoints, int k, double scale, uint64_t seed, mlmq_host_graph **out) {
    if (!out || npoints < 2 || k < 1 || k >= npoints || k > 16 || !(scale > 0))
        return MLMQ_ERR_ARG;
    auto *g = new (std::nothrow) mlmq_host_graph;
    if (!g) return MLMQ_ERR_NOMEM;
    try {
        const int n = npoints;
        std::vector<double> px(n), py(n);
        for (int i = 0; i < n; i++) {
            px[i] = unit01(hash3(seed, 1, (uint64_t)i));
            py[i] = unit01(hash3(seed, 2, (uint64_t)i));
        }
        // About two points per cell; cells ordered by Morton code.
        int G = std::max(1, (int)std::sqrt(n / 2.0));
        if (G > 65535) G = 65535;
        auto cellx = [&](double x) { return std::min(G - 1, (int)(x * G)); };
        std::vector<uint64_t> key(n);
        for (int i = 0; i < n; i++) {
            uint32_t cx = (uint32_t)cellx(px[i]), cy = (uint32_t)cellx(py[i]);
            key[i] = ((uint64_t)(morton16(cx) | (morton16(cy) << 1)) << 32) | (uint32_t)i;
        }
        std::sort(key.begin(), key.end());
        g->perm.resize(n);
        std::vector<double> x(n), y(n);
        for (int v = 0; v < n; v++) {
            int i = (int)(key[v] & 0xffffffffu);
            g->perm[v] = i;
            x[v] = px[i];
            y[v] = py[i];
        }
        std::vector<int> cbeg((size_t)G * G, 0), cend((size_t)G * G, 0);
        for (int v = 0; v < n; v++) {
            size_t c = (size_t)cellx(y[v]) * G + cellx(x[v]);
            if (cend[c] == 0) cbeg[c] = v;
            cend[c] = v + 1;
        }
        const double cs = 1.0 / G;
        std::vector<int> nbr((size_t)n * k);
        parallel_for(n, [&](int64_t b, int64_t e, int) {
            std::vector<std::pair<double, int>> best;
            for (int64_t v = b; v < e; v++) {
                best.clear();
                int cx = cellx(x[v]), cy = cellx(y[v]);
                for (int r = 0;; r++) {
                    for (int yy = cy - r; yy <= cy + r; yy++) {
                        if (yy < 0 || yy >= G) continue;
                        bool edge_row = (yy == cy - r || yy == cy + r);
                        for (int xx = cx - r; xx <= cx + r; xx += (edge_row ? 1 : 2 * r)) {
                            if (xx >= 0 && xx < G) {
                                size_t c = (size_t)yy * G + xx;
                                for (int u = cbeg[c]; u < cend[c]; u++) {
                                    if (u == v) continue;
                                    double dx = x[u] - x[v], dy = y[u] - y[v];
                                    best.emplace_back(dx * dx + dy * dy, u);
                                }
                            }
                            if (r == 0) break;
                        }
                    }
                    if ((int)best.size() >= k) {
                        std::partial_sort(best.begin(), best.begin() + k, best.end());
                        best.resize(k);
                        double lim = r * cs;
                        if (best[k - 1].first <= lim * lim) break;
                    }
                    if (r > 2 * G) break;
                }
                for (int j = 0; j < k; j++) nbr[(size_t)v * k + j] = best[j].second;
            }
        });
        std::vector<uint64_t> pairs;
        pairs.reserve((size_t)n * k);
        for (int v = 0; v < n; v++)
            for (int j = 0; j < k; j++) {
                int u = nbr[(size_t)v * k + j];
                int a = std::min(u, v), c = std::max(u, v);
                pairs.push_back(((uint64_t)a << 32) | (uint32_t)c);
            }
        std::sort(pairs.begin(), pairs.end());
        pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
        std::vector<int> pw(pairs.size());
        for (size_t i = 0; i < pairs.size(); i++) {
            int a = (int)(pairs[i] >> 32), c = (int)(pairs[i] & 0xffffffffu);
            double dx = x[a] - x[c], dy = y[a] - y[c];
            double wd = std::llround(scale * std::sqrt(dx * dx + dy * dy)) + 1.0;
            if (wd >= INT_MAX) throw std::bad_alloc();
            pw[i] = (int)wd;
        }
        int rc = csr_from_pairs(n, pairs, pw, *g);
        if (rc) {
            delete g;
            return rc;
        }
    } catch (...) {
        delete g;
        return MLMQ_ERR_NOMEM;
    }
    *out = g;
    return MLMQ_OK;
}

int mlmq_hgraph_rmat(int scale, int edge_factor, double a, double b, double c, int wmin, int wmax,
                     uint64_t seed, mlmq_host_graph **out) {
    if (!out || scale < 1 || scale > 30 || edge_factor < 1 || a < 0 || b < 0 || c < 0 ||
        a + b + c > 1 || wmin < 0 || wmax < wmin)
        return MLMQ_ERR_ARG;
    int64_t n64 = (int64_t)1 << scale;
    int64_t samples = n64 * edge_factor;
    if (n64 >= INT_MAX || samples >= INT_MAX) return MLMQ_ERR_RANGE;
    auto *g = new (std::nothrow) mlmq_host_graph;
    if (!g) return MLMQ_ERR_NOMEM;
    try {
        const int n = (int)n64;
        // Quadrant thresholds on a 16-bit uniform draw per level.
        const uint32_t ta = (uint32_t)std::llround(a * 65536.0);
        const uint32_t tb = (uint32_t)std::llround((a + b) * 65536.0);
        const uint32_t tc = (uint32_t)std::llround((a + b + c) * 65536.0);
        std::vector<int> su((size_t)samples), sv((size_t)samples);
        parallel_for(samples, [&](int64_t lo, int64_t hi, int) {
            for (int64_t i = lo; i < hi; i++) {
                uint32_t u = 0, v = 0;
                uint64_t h = 0;
                for (int lvl = 0; lvl < scale; lvl++) {
                    if ((lvl & 3) == 0) h = hash3(seed, 3, (uint64_t)i * 8 + (uint64_t)(lvl >> 2));
                    uint32_t r = (uint32_t)(h & 0xffff);
                    h >>= 16;
                    uint32_t bu = r >= tb, bv = (r >= ta && r < tb) || r >= tc;
                    u = (u << 1) | bu;
                    v = (v << 1) | bv;
                }
                su[i] = (int)u;
                sv[i] = (int)v;
            }
        });
        // Bucket by source (counting sort), then sort/unique each row.
        std::vector<int> deg((size_t)n + 1, 0);
        for (int64_t i = 0; i < samples; i++)
            if (su[i] != sv[i]) deg[su[i] + 1]++;
        for (int i = 0; i < n; i++) deg[i + 1] += deg[i];
        std::vector<int> tmp((size_t)deg[n]);
        {
            std::vector<int> fill(deg.begin(), deg.end() - 1);
            for (int64_t i = 0; i < samples; i++)
                if (su[i] != sv[i]) tmp[fill[su[i]]++] = sv[i];
        }
        std::vector<int>().swap(su);
        std::vector<int>().swap(sv);
        std::vector<int> keepn((size_t)n, 0);
        parallel_for(n, [&](int64_t lo, int64_t hi, int) {
            for (int64_t u = lo; u < hi; u++) {
                auto bgn = tmp.begin() + deg[u], end = tmp.begin() + deg[u + 1];
                std::sort(bgn, end);
                keepn[u] = (int)(std::unique(bgn, end) - bgn);
            }
        });
        g->n = n;
        g->row.assign((size_t)n + 1, 0);
        for (int u = 0; u < n; u++) g->row[u + 1] = g->row[u] + keepn[u];
        g->m = g->row[n];
        g->col.resize((size_t)g->m);
        g->w.resize((size_t)g->m);
        parallel_for(n, [&](int64_t lo, int64_t hi, int) {
            for (int64_t u = lo; u < hi; u++)
                for (int j = 0; j < keepn[u]; j++) {
                    int v = tmp[deg[u] + j];
                    int p = g->row[u] + j;
                    g->col[p] = v;
                    g->w[p] = uniform_int(hash3(seed, 4, ((uint64_t)u << 32) | (uint32_t)v), wmin,
                                          wmax);
                }
        });
    } catch (...) {
        delete g;
        return MLMQ_ERR_NOMEM;
    }
    *out = g;
    return MLMQ_OK;
}

int mlmq_hgraph_from_csr(int n, int64_t m, const int *row, const int *col, const int *w,
                         mlmq_host_graph **out) {
    if (!out) return MLMQ_ERR_ARG;
    int rc = validate_csr(n, m, row, col, w);
    if (rc) return rc;
    auto *g = new (std::nothrow) mlmq_host_graph;
    if (!g) return MLMQ_ERR_NOMEM;
    try {
        g->n = n;
        g->m = m;
        g->row.assign(row, row + n + 1);
        g->col.assign(col, col + m);
        g->w.assign(w, w + m);
    } catch (...) {
        delete g;
        return MLMQ_ERR_NOMEM;
    }
    *out = g;
    return MLMQ_OK;
}

int mlmq_hgraph_read_gr(const char *path, mlmq_host_graph **out) {
    if (!path || !out) return MLMQ_ERR_ARG;
    int fd = open(path, O_RDONLY);
    if (fd < 0) return MLMQ_ERR_IO;
    struct stat st;
    if (fstat(fd, &st) != 0 || st.st_size < 32) {
        close(fd);
        return MLMQ_ERR_IO;
    }
    size_t bytes = (size_t)st.st_size;
    void *p = mmap(nullptr, bytes, PROT_READ, MAP_PRIVATE, fd, 0);
    close(fd);
    if (p == MAP_FAILED) return MLMQ_ERR_IO;
    const uint64_t *h = (const uint64_t *)p;
    int rc = MLMQ_OK;
    mlmq_host_graph *g = nullptr;
    do {
        if (h[0] != 1 || h[1] != 4 || h[2] == 0 || h[2] >= INT_MAX || h[3] >= INT_MAX) {
            rc = MLMQ_ERR_IO;
            break;
        }
        uint64_t n = h[2], m = h[3];
        if (bytes < 32 + 8 * n + 8 * m + 4 * (m & 1)) {
            rc = MLMQ_ERR_IO;
            break;
        }
        const uint64_t *ends = h + 4;
        const uint32_t *dst = (const uint32_t *)(ends + n);
        const int32_t *wt = (const int32_t *)(dst + m + (m & 1));
        g = new (std::nothrow) mlmq_host_graph;
        if (!g) {
            rc = MLMQ_ERR_NOMEM;
            break;
        }
        try {
            g->n = (int)n;
            g->m = (int64_t)m;
            g->row.assign(n + 1, 0);
            for (uint64_t u = 0; u < n; u++) {
                if (ends[u] > m || (u && ends[u] < ends[u - 1])) {
                    rc = MLMQ_ERR_IO;
                    break;
                }
                g->row[u + 1] = (int)ends[u];
            }
            if (!rc && (uint64_t)g->row[n] != m) rc = MLMQ_ERR_IO;
            if (!rc) {
                g->col.assign((const int *)dst, (const int *)dst + m);
                g->w.assign(wt, wt + m);
                for (uint64_t e = 0; e < m; e++)
                    if (g->col[e] < 0 || (uint64_t)g->col[e] >= n || g->w[e] < 0) {
                        rc = MLMQ_ERR_IO;
                        break;
                    }
            }
        } catch (...) {
            rc = MLMQ_ERR_NOMEM;
        }
    } while (0);
    munmap(p, bytes);
    if (rc) {
        delete g;
        return rc;
    }
    *out = g;
    return MLMQ_OK;
}

int mlmq_hgraph_write_gr(const mlmq_host_graph *g, const char *path) {
    if (!g || !path) return MLMQ_ERR_ARG;
    FILE *f = fopen(path, "wb");
    if (!f) return MLMQ_ERR_IO;
    uint64_t hdr[4] = {1, 4, (uint64_t)g->n, (uint64_t)g->m};
    bool ok = fwrite(hdr, sizeof(hdr), 1, f) == 1;
    std::vector<uint64_t> ends((size_t)g->n);
    for (int u = 0; u < g->n; u++) ends[u] = (uint64_t)g->row[u + 1];
    ok = ok && fwrite(ends.data(), 8, ends.size(), f) == ends.size();
    ok = ok && fwrite(g->col.data(), 4, (size_t)g->m, f) == (size_t)g->m;
    uint32_t zero = 0;
    if (g->m & 1) ok = ok && fwrite(&zero, 4, 1, f) == 1;
    ok = ok && fwrite(g->w.data(), 4, (size_t)g->m, f) == (size_t)g->m;
    ok = (fclose(f) == 0) && ok;
    return ok ? MLMQ_OK : MLMQ_ERR_IO;
}

int mlmq_hgraph_view(const mlmq_host_graph *g, int *n, int64_t *m, const int **row,
                     const int **col, const int **w, const int **perm) {
    if (!g) return MLMQ_ERR_ARG;
    if (n) *n = g->n;
    if (m) *m = g->m;
    if (row) *row = g->row.data();
    if (col) *col = g->col.data();
    if (w) *w = g->w.data();
    if (perm) *perm = g->perm.empty() ? nullptr : g->perm.data();
    return MLMQ_OK;
}

void mlmq_hgraph_free(mlmq_host_graph *g) { delete g; }

// BFS locality order (reference graph_transform/reorder_gr.cu:96-130,
// 161-190): vertices numbered in the discovery order of a queue BFS from
// `root` that scans arcs in CSR order; vertices never reached follow in
// ascending original id.  Rows keep their arcs in the original order with the
// destinations renumbered.  perm[new] = old and invperm[old] = new (each n
// entries, optional).
int mlmq_hgraph_reorder_bfs(const mlmq_host_graph *g, int root, mlmq_host_graph **out, int *perm,
                            int *invperm) {
    if (!g || !out || root < 0 || root >= g->n) return MLMQ_ERR_ARG;
    auto *r = new (std::nothrow) mlmq_host_graph;
    if (!r) return MLMQ_ERR_NOMEM;
    try {
        const int n = g->n;
        std::vector<int> p((size_t)n), inv((size_t)n, -1), q((size_t)n);
        int head = 0, tail = 0, next = 0;
        q[tail++] = root;
        inv[root] = next;
        p[next++] = root;
        while (head < tail) {
            const int u = q[head++];
            for (int e = g->row[u]; e < g->row[u + 1]; e++) {
                const int v = g->col[e];
                if (inv[v] == -1) {
                    inv[v] = next;
                    p[next++] = v;
                    q[tail++] = v;
                }
            }
        }
        for (int v = 0; v < n; v++)
            if (inv[v] == -1) {
                inv[v] = next;
                p[next++] = v;
            }
        r->n = n;
        r->m = g->m;
        r->row.assign((size_t)n + 1, 0);
        for (int i = 0; i < n; i++) r->row[i + 1] = r->row[i] + (g->row[p[i] + 1] - g->row[p[i]]);
        r->col.resize((size_t)g->m);
        r->w.resize((size_t)g->m);
        parallel_for(n, [&](int64_t b, int64_t e, int) {
            for (int64_t i = b; i < e; i++) {
                int pos = r->row[i];
                for (int a = g->row[p[i]]; a < g->row[p[i] + 1]; a++, pos++) {
                    r->col[pos] = inv[g->col[a]];
                    r->w[pos] = g->w[a];
                }
            }
        });
        if (perm) std::copy(p.begin(), p.end(), perm);
        if (invperm) std::copy(inv.begin(), inv.end(), invperm);
    } catch (...) {
        delete r;
        return MLMQ_ERR_NOMEM;
    }
    *out = r;
    return MLMQ_OK;
}

// Chain-shortcut augmentation G+.  The graph it produces is the one the
// reference's builder produces (SSSP/l3/l3_chain_shortcuts.h:23-109, strict
// variant): the same chain vertices, the same shortcut arcs in the same
// order, the same statistics -- tests compare both byte for byte.  The way
// it gets there is data-parallel:
//
//  1. Chain vertices, one independent test per vertex: not the source,
//     exactly two out-arcs to two distinct other vertices on its own side of
//     `cut`, in-degree exactly two, and an arc back from each of its two
//     out-neighbours (so its two in-arcs come from exactly those vertices).
//  2. Walks through chains by pointer jumping.  A "step" is an out-arc of a
//     chain vertex: (c, k) = the k-th out-arc of c, to y.  When y is a chain
//     vertex the walk continues on y's out-arc that does not return to c;
//     otherwise the step ends the walk.  Every step starts with its own arc
//     (weight, one hop, end y) and a link to its successor; each round,
//     every step adds its successor's totals and links to the successor's
//     successor, so after ceil(log2 L) rounds every step knows the weight,
//     hop count and end of the rest of its walk (Wyllie's list ranking).
//     Steps on a closed ring of chain vertices never finish; no walk from a
//     non-chain vertex can enter such a ring.
//  3. From every non-chain vertex u, out-arc f to a chain vertex c continues
//     on c's step away from u: weight w(f) + the step's total, hops 1 + its
//     hops.  One shortcut u -> end per such walk that does not come back to
//     u and whose weight stays below INT_MAX, placed before u's original arcs
//     in the order of u's out-arcs.  Every original arc is kept, so
//     shortest-path distances are unchanged.
//
// stats (optional, 5 entries): chain vertices, shortcuts, longest walk in
// arcs, walks dropped for overflow, arcs the shortcuts stand for.
int mlmq_hgraph_chain_shortcuts(const mlmq_host_graph *g, int cut, int source,
                                mlmq_host_graph **out, int64_t *stats) {
    if (!g || !out) return MLMQ_ERR_ARG;
    const int n = g->n;
    if (source < 0 || source >= n || cut < 0 || cut > n) return MLMQ_ERR_ARG;
    auto *r = new (std::nothrow) mlmq_host_graph;
    if (!r) return MLMQ_ERR_NOMEM;
    int rc = MLMQ_OK;
    try {
        const int *row = g->row.data(), *dst = g->col.data(), *wt = g->w.data();
        // ---- 1. chain vertices ------------------------------------------------
        std::vector<std::atomic<int>> indeg((size_t)n);
        parallel_for(n, [&](int64_t b, int64_t e, int) {
            for (int64_t v = b; v < e; v++) indeg[v].store(0, std::memory_order_relaxed);
        });
        parallel_for(g->m, [&](int64_t b, int64_t e, int) {
            for (int64_t a = b; a < e; a++) indeg[dst[a]].fetch_add(1, std::memory_order_relaxed);
        });
        auto has_arc = [&](int from, int to) {
            for (int a = row[from]; a < row[from + 1]; a++)
                if (dst[a] == to) return true;
            return false;
        };
        std::vector<int> chain_id((size_t)n, -1);  // compact index of each chain vertex
        std::vector<unsigned char> is_chain((size_t)n, 0);
        parallel_for(n, [&](int64_t b, int64_t e, int) {
            for (int64_t vv = b; vv < e; vv++) {
                const int v = (int)vv;
                if (v == source || row[v + 1] - row[v] != 2 || indeg[v].load() != 2) continue;
                const int x = dst[row[v]], y = dst[row[v] + 1];
                const bool side = v < cut;
                if (x == v || y == v || x == y || (x < cut) != side || (y < cut) != side) continue;
                is_chain[v] = has_arc(x, v) && has_arc(y, v);
            }
        });
        int nchain = 0;
        for (int v = 0; v < n; v++)
            if (is_chain[v]) chain_id[v] = nchain++;
        // ---- 2. pointer jumping over chain steps ------------------------------
        // Step 2*chain_id[c] + k is c's k-th out-arc.
        const int64_t steps = 2 * (int64_t)nchain;
        std::vector<int64_t> len((size_t)steps), len2((size_t)steps);
        std::vector<int> hop((size_t)steps), hop2((size_t)steps);
        std::vector<int> end((size_t)steps), end2((size_t)steps);
        std::vector<int> nxt((size_t)steps), nxt2((size_t)steps);
        // The step of chain vertex c that leaves along the arc not going to `from`.
        auto away_from = [&](int c, int from) -> int64_t {
            return 2 * (int64_t)chain_id[c] + (dst[row[c]] == from ? 1 : 0);
        };
        parallel_for(n, [&](int64_t b, int64_t e, int) {
            for (int64_t cc = b; cc < e; cc++) {
                const int c = (int)cc;
                if (!is_chain[c]) continue;
                for (int k = 0; k < 2; k++) {
                    const int64_t s = 2 * (int64_t)chain_id[c] + k;
                    const int a = row[c] + k, y = dst[a];
                    len[s] = wt[a];
                    hop[s] = 1;
                    end[s] = y;
                    nxt[s] = is_chain[y] ? (int)away_from(y, c) : -1;
                }
            }
        });
        int rounds = 1;
        while (((int64_t)1 << rounds) <= steps) rounds++;
        for (int it = 0; it <= rounds; it++) {
            std::atomic<bool> live(false);
            parallel_for(steps, [&](int64_t b, int64_t e, int) {
                bool any = false;
                for (int64_t s = b; s < e; s++) {
                    const int t = nxt[s];
                    if (t < 0) {
                        len2[s] = len[s];
                        hop2[s] = hop[s];
                        end2[s] = end[s];
                        nxt2[s] = -1;
                        continue;
                    }
                    // Weights are below 2^31 and a walk has fewer than 2^31
                    // arcs, so the sum fits in 63 bits.
                    len2[s] = len[s] + len[t];
                    hop2[s] = hop[s] + hop[t];
                    end2[s] = end[t];
                    nxt2[s] = nxt[t];
                    any = any || nxt[t] >= 0;
                }
                if (any) live.store(true);
            });
            len.swap(len2);
            hop.swap(hop2);
            end.swap(end2);
            nxt.swap(nxt2);
            if (!live.load()) break;
        }
        // ---- 3. shortcuts from non-chain vertices -----------------------------
        // Per out-arc of a non-chain vertex: 0 no shortcut, 1 shortcut,
        // 2 dropped for overflow.
        std::vector<unsigned char> kind((size_t)g->m, 0);
        std::vector<int> count((size_t)n + 1, 0);
        std::atomic<int> bad(0);
        parallel_for(n, [&](int64_t b, int64_t e, int) {
            for (int64_t uu = b; uu < e; uu++) {
                const int u = (int)uu;
                int c = row[u + 1] - row[u];
                if (!is_chain[u])
                    for (int f = row[u]; f < row[u + 1]; f++) {
                        const int h = dst[f];
                        if (!is_chain[h]) continue;
                        const int64_t s = away_from(h, u);
                        if (nxt[s] >= 0) {  // cannot happen: walks from u end
                            bad.store(1);
                            continue;
                        }
                        if ((int64_t)wt[f] + len[s] >= INT_MAX) {
                            kind[f] = 2;
                            continue;
                        }
                        if (end[s] == u) continue;
                        if ((end[s] < cut) != (u < cut)) bad.store(1);
                        kind[f] = 1;
                        c++;
                    }
                count[u + 1] = c;
            }
        });
        if (bad.load()) rc = MLMQ_ERR_ARG;
        int64_t total = 0;
        for (int u = 0; u < n && !rc; u++) {
            total += count[u + 1];
            if (total >= INT_MAX) rc = MLMQ_ERR_RANGE;
        }
        if (!rc) {
            r->n = n;
            r->m = total;
            r->row.assign((size_t)n + 1, 0);
            for (int u = 0; u < n; u++) r->row[u + 1] = r->row[u] + count[u + 1];
            r->col.resize((size_t)total);
            r->w.resize((size_t)total);
            std::vector<int64_t> part(4 * (size_t)num_threads() + 4, 0);  // per thread: shortcuts,
                                                                       // longest, overflow, arcs
            parallel_for(n, [&](int64_t b, int64_t e, int t) {
                int64_t ns = 0, lg = 0, ov = 0, ar = 0;
                for (int64_t uu = b; uu < e; uu++) {
                    const int u = (int)uu;
                    int p = r->row[u];
                    for (int f = row[u]; f < row[u + 1]; f++) {
                        if (kind[f] == 2) ov++;
                        if (kind[f] != 1) continue;
                        const int64_t s = away_from(dst[f], u);
                        r->col[p] = end[s];
                        r->w[p++] = (int)(wt[f] + len[s]);
                        const int64_t hops = 1 + (int64_t)hop[s];
                        ns++;
                        ar += hops;
                        lg = std::max(lg, hops);
                    }
                    for (int f = row[u]; f < row[u + 1]; f++) {
                        r->col[p] = dst[f];
                        r->w[p++] = wt[f];
                    }
                }
                part[4 * (size_t)t] = ns;
                part[4 * (size_t)t + 1] = lg;
                part[4 * (size_t)t + 2] = ov;
                part[4 * (size_t)t + 3] = ar;
            });
            if (stats) {
                int64_t ns = 0, lg = 0, ov = 0, ar = 0;
                for (size_t t = 0; t + 3 < part.size(); t += 4) {
                    ns += part[t];
                    lg = std::max(lg, part[t + 1]);
                    ov += part[t + 2];
                    ar += part[t + 3];
                }
                stats[0] = nchain;
                stats[1] = ns;
                stats[2] = lg;
                stats[3] = ov;
                stats[4] = ar;
            }
        }
    } catch (...) {
        rc = MLMQ_ERR_NOMEM;
    }
    if (rc) {
        delete r;
        return rc;
    }
    *out = r;
    return MLMQ_OK;
}

}  // extern "C"
