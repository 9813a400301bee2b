// reorder.cu -- BFS locality reordering as a device preprocessing step.
//
// The order is the reference tool's (graph_transform/reorder_gr.cu:96-190):
// new ids follow the discovery order of a FIFO breadth-first search from
// `root` that scans each vertex's arcs in CSR order; vertices the search
// never reaches follow in ascending id.  Each new row keeps its old row's
// arcs in order, destinations renamed.  The output equals the host
// implementation (mlmq_hgraph_reorder_bfs) byte for byte.
//
// A FIFO search discovers the vertices of one level in the order of their
// first discovering arc: (queue position of the parent, index of the arc in
// the parent's row).  The device search is level-synchronous and reproduces
// that order exactly:
//   1. every arc out of the current level's vertices (queue positions
//      [lo, hi), which ARE their new ids) proposes the key
//      position << 32 | arc index to its undiscovered target with a 64-bit
//      atomicMin; the first proposal to a target also appends it to the
//      level's candidate list;
//   2. the candidates are sorted by key (CUB radix sort): that is their
//      discovery order, so candidate i gets new id hi + i;
//   3. the next level is [hi, hi + count).
// Then the unreached vertices are appended in ascending id (CUB select), the
// new row offsets are a scan of the permuted degrees, and one warp per new
// row copies and renames its arcs.  Everything stays on the device; the
// host reads one count per level.
#include "host_graph.h"
#include "mlmq_b200.h"
#include "solver_internal.h"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <climits>
#include <new>

namespace mlmq {
namespace {

constexpr unsigned long long NO_KEY = ~0ull;

__global__ void reorder_init_kernel(int n, int *inv, unsigned long long *key, int *mark) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        inv[v] = -1;
        key[v] = NO_KEY;
        mark[v] = -1;
    }
}

__global__ void reorder_seed_kernel(int root, int *inv, int *perm) {
    inv[root] = 0;
    perm[0] = root;
}

// One warp per vertex of the current level: its lanes stride the row.
__global__ void reorder_discover_kernel(const int *__restrict__ row, const int *__restrict__ col,
                                        const int *__restrict__ perm, int lo, int hi, int level,
                                        const int *__restrict__ inv, unsigned long long *key,
                                        int *mark, int *cand, int *count) {
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long p = lo + ((long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5));
         p < hi; p += warps) {
        const int u = perm[p];
        const int beg = row[u], deg = row[u + 1] - beg;
        for (int j = lane; j < deg; j += 32) {
            const int v = col[beg + j];
            if (inv[v] >= 0) continue;  // discovered at an earlier level
            const unsigned long long k = ((unsigned long long)p << 32) | (unsigned)j;
            if (k < key[v]) atomicMin(key + v, k);
            if (atomicExch(mark + v, level) != level) cand[atomicAdd(count, 1)] = v;
        }
    }
}

__global__ void reorder_gather_keys_kernel(const int *__restrict__ cand, int c,
                                           unsigned long long *key, unsigned long long *ck) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < c; i += gridDim.x * blockDim.x) {
        const int v = cand[i];
        ck[i] = key[v];
        key[v] = NO_KEY;
    }
}

__global__ void reorder_assign_kernel(const int *__restrict__ sorted, int c, int base, int *inv,
                                      int *perm) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < c; i += gridDim.x * blockDim.x) {
        const int v = sorted[i];
        inv[v] = base + i;
        perm[base + i] = v;
    }
}

struct Unreached {
    const int *inv;
    __device__ bool operator()(int v) const { return inv[v] < 0; }
};

__global__ void reorder_tail_kernel(const int *__restrict__ left, const int *__restrict__ nleft,
                                    int base, int *inv, int *perm) {
    const int c = *nleft;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < c; i += gridDim.x * blockDim.x) {
        const int v = left[i];
        inv[v] = base + i;
        perm[base + i] = v;
    }
}

__global__ void reorder_degree_kernel(const int *__restrict__ row, const int *__restrict__ perm,
                                      int n, int *deg_out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int v = perm[i];
        deg_out[i + 1] = row[v + 1] - row[v];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) deg_out[0] = 0;
}

__global__ void reorder_fill_kernel(const int *__restrict__ row, const int *__restrict__ col,
                                    const int *__restrict__ w, const int *__restrict__ perm,
                                    const int *__restrict__ inv, const int *__restrict__ row_out,
                                    int n, int *col_out, int *w_out) {
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long i = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n;
         i += warps) {
        const int v = perm[i];
        const int beg = row[v], deg = row[v + 1] - beg, out = row_out[i];
        for (int j = lane; j < deg; j += 32) {
            col_out[out + j] = inv[col[beg + j]];
            w_out[out + j] = w[beg + j];
        }
    }
}

int grid_for(long long items, int per_block) {
    const long long b = (items + per_block - 1) / per_block;
    return (int)std::max(1ll, std::min(b, 148ll * 32));
}

}  // namespace
}  // namespace mlmq

using namespace mlmq;

extern "C" int mlmq_reorder_bfs_device(int n, int64_t m, const int *d_row, const int *d_col,
                                       const int *d_w, int root, int *d_row_out, int *d_col_out,
                                       int *d_w_out, int *d_perm, int *d_invperm, void *stream) {
    if (n <= 0 || m < 0 || m >= INT_MAX || !d_row || (m > 0 && (!d_col || !d_w)) || root < 0 ||
        root >= n || !d_row_out || (m > 0 && (!d_col_out || !d_w_out)) || !d_perm || !d_invperm)
        return MLMQ_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    int *inv = d_invperm, *perm = d_perm;
    unsigned long long *key = nullptr, *ck = nullptr, *ck_sorted = nullptr;
    int *mark = nullptr, *cand = nullptr, *cand_sorted = nullptr, *count = nullptr;
    int *h_count = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    int rc = MLMQ_OK;
    const size_t N = (size_t)n;
    if (!rc) rc = dev_alloc(&key, 8 * N, st, "reorder keys");
    if (!rc) rc = dev_alloc(&ck, 8 * N, st, "reorder level keys");
    if (!rc) rc = dev_alloc(&ck_sorted, 8 * N, st, "reorder sorted keys");
    if (!rc) rc = dev_alloc(&mark, 4 * N, st, "reorder marks");
    if (!rc) rc = dev_alloc(&cand, 4 * N, st, "reorder candidates");
    if (!rc) rc = dev_alloc(&cand_sorted, 4 * N, st, "reorder sorted candidates");
    if (!rc) rc = dev_alloc(&count, 64, st, "reorder count");
    if (!rc) rc = pinned_alloc(&h_count, 64);
    // One temporary buffer for every CUB call: the largest need.
    if (!rc) {
        size_t a = 0, b = 0, c = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, a, ck, ck_sorted, cand, cand_sorted, n, 0, 64, st);
        cub::DeviceSelect::If(nullptr, b, thrust::counting_iterator<int>(0), cand, count, n,
                              Unreached{inv}, st);
        cub::DeviceScan::InclusiveSum(nullptr, c, reinterpret_cast<int *>(ck), d_row_out, n + 1, st);
        tmp_bytes = std::max(a, std::max(b, c));
        rc = dev_alloc(&tmp, tmp_bytes, st, "reorder temporary");
    }
    if (!rc) {
        reorder_init_kernel<<<grid_for(n, 256), 256, 0, st>>>(n, inv, key, mark);
        reorder_seed_kernel<<<1, 1, 0, st>>>(root, inv, perm);
        rc = cuda_fail(cudaGetLastError(), "reorder init");
    }
    int lo = 0, hi = 1;
    for (int level = 0; !rc && lo < hi; level++) {
        rc = cuda_fail(cudaMemsetAsync(count, 0, sizeof(int), st), "reorder count reset");
        if (rc) break;
        reorder_discover_kernel<<<grid_for((long long)(hi - lo) * 32, 256), 256, 0, st>>>(
            d_row, d_col, perm, lo, hi, level, inv, key, mark, cand, count);
        rc = cuda_fail(cudaGetLastError(), "reorder discover");
        if (!rc) rc = cuda_fail(cudaMemcpyAsync(h_count, count, sizeof(int), cudaMemcpyDeviceToHost, st),
                                "reorder count");
        if (!rc) rc = cuda_fail(cudaStreamSynchronize(st), "reorder level");
        if (rc) break;
        const int c = *h_count;
        if (c <= 0) break;
        reorder_gather_keys_kernel<<<grid_for(c, 256), 256, 0, st>>>(cand, c, key, ck);
        size_t tb = tmp_bytes;
        rc = cuda_fail(cub::DeviceRadixSort::SortPairs(tmp, tb, ck, ck_sorted, cand, cand_sorted, c, 0,
                                                       64, st), "reorder sort");
        if (rc) break;
        reorder_assign_kernel<<<grid_for(c, 256), 256, 0, st>>>(cand_sorted, c, hi, inv, perm);
        rc = cuda_fail(cudaGetLastError(), "reorder assign");
        lo = hi;
        hi += c;
    }
    if (!rc && hi < n) {
        // Unreached vertices in ascending id.
        size_t tb = tmp_bytes;
        rc = cuda_fail(cub::DeviceSelect::If(tmp, tb, thrust::counting_iterator<int>(0), cand, count,
                                             n, Unreached{inv}, st), "reorder unreached");
        if (!rc) {
            reorder_tail_kernel<<<grid_for(n - hi, 256), 256, 0, st>>>(cand, count, hi, inv, perm);
            rc = cuda_fail(cudaGetLastError(), "reorder tail");
        }
    }
    if (!rc) {
        // Degrees of the new rows (8n bytes of ck hold n + 1 ints), then
        // their inclusive sum with a leading 0: the new row offsets.
        int *deg = reinterpret_cast<int *>(ck);
        reorder_degree_kernel<<<grid_for(n, 256), 256, 0, st>>>(d_row, perm, n, deg);
        size_t tb = tmp_bytes;
        rc = cuda_fail(cub::DeviceScan::InclusiveSum(tmp, tb, deg, d_row_out, n + 1, st),
                       "reorder offsets");
    }
    if (!rc && m > 0) {
        reorder_fill_kernel<<<grid_for((long long)n * 32, 256), 256, 0, st>>>(
            d_row, d_col, d_w, perm, inv, d_row_out, n, d_col_out, d_w_out);
        rc = cuda_fail(cudaGetLastError(), "reorder fill");
    }
    if (!rc) rc = cuda_fail(cudaStreamSynchronize(st), "reorder");
    dev_free(key, st);
    dev_free(ck, st);
    dev_free(ck_sorted, st);
    dev_free(mark, st);
    dev_free(cand, st);
    dev_free(cand_sorted, st);
    dev_free(count, st);
    dev_free(tmp, st);
    pinned_free(h_count, 64);
    return rc;
}

extern "C" int mlmq_hgraph_reorder_bfs_gpu(const mlmq_host_graph *g, int root, mlmq_host_graph **out,
                                           int *perm, int *invperm) {
    if (!g || !out || root < 0 || root >= g->n) return MLMQ_ERR_ARG;
    const int n = g->n;
    const int64_t m = g->m;
    auto *r = new (std::nothrow) mlmq_host_graph;
    if (!r) return MLMQ_ERR_NOMEM;
    cudaStream_t st = nullptr;
    int rc = cuda_fail(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "reorder stream");
    int *d[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    const size_t sz[8] = {(size_t)n + 1, (size_t)m, (size_t)m, (size_t)n + 1, (size_t)m, (size_t)m,
                          (size_t)n, (size_t)n};
    for (int i = 0; i < 8 && !rc; i++) rc = dev_alloc(&d[i], 4 * std::max<size_t>(sz[i], 1), st, "reorder buffers");
    try {
        r->n = n;
        r->m = m;
        r->row.resize((size_t)n + 1);
        r->col.resize((size_t)m);
        r->w.resize((size_t)m);
    } catch (...) {
        rc = rc ? rc : MLMQ_ERR_NOMEM;
    }
    if (!rc) rc = cuda_fail(cudaMemcpyAsync(d[0], g->row.data(), 4 * sz[0], cudaMemcpyHostToDevice, st), "H2D row");
    if (!rc && m) rc = cuda_fail(cudaMemcpyAsync(d[1], g->col.data(), 4 * sz[1], cudaMemcpyHostToDevice, st), "H2D col");
    if (!rc && m) rc = cuda_fail(cudaMemcpyAsync(d[2], g->w.data(), 4 * sz[2], cudaMemcpyHostToDevice, st), "H2D w");
    if (!rc) rc = mlmq_reorder_bfs_device(n, m, d[0], d[1], d[2], root, d[3], d[4], d[5], d[6], d[7], st);
    if (!rc) rc = cuda_fail(cudaMemcpyAsync(r->row.data(), d[3], 4 * sz[3], cudaMemcpyDeviceToHost, st), "D2H row");
    if (!rc && m) rc = cuda_fail(cudaMemcpyAsync(r->col.data(), d[4], 4 * sz[4], cudaMemcpyDeviceToHost, st), "D2H col");
    if (!rc && m) rc = cuda_fail(cudaMemcpyAsync(r->w.data(), d[5], 4 * sz[5], cudaMemcpyDeviceToHost, st), "D2H w");
    if (!rc && perm) rc = cuda_fail(cudaMemcpyAsync(perm, d[6], 4 * (size_t)n, cudaMemcpyDeviceToHost, st), "D2H perm");
    if (!rc && invperm) rc = cuda_fail(cudaMemcpyAsync(invperm, d[7], 4 * (size_t)n, cudaMemcpyDeviceToHost, st), "D2H invperm");
    if (st) {
        const int src = cuda_fail(cudaStreamSynchronize(st), "reorder copies");
        if (!rc) rc = src;
    }
    for (int i = 0; i < 8; i++) dev_free(d[i], st);
    if (st) cudaStreamDestroy(st);
    if (rc) {
        delete r;
        return rc;
    }
    *out = r;
    return MLMQ_OK;
}
