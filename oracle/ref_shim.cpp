// oracle/ref_shim.cpp -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// Wraps the reference's own CPU Dijkstra, `sssp_sequential` from
// evidence/l3_supplement_20260921_v2/single_source/SSSP/main.cu:47-117, which
// oracle/Makefile compiles unchanged from the reference tree (with its `main`
// renamed so the object can live in a shared library), behind a C entry point
// that tests and bench.py's CPU-baseline leg load with ctypes.
//
// main.cu also references the GPU solver entry points that its own main()
// calls (main.cu:15-17).  The checker never runs that main(), so the three
// definitions below only satisfy the dynamic loader; each returns -1.
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "common.h"
#include "graph_info.h"

void sssp_sequential(int m, int nnz, int *RowPtr, int *ColIdx, VALUE_TYPE *edge_data,
                     VALUE_TYPE *node_data, int *prep, int *hop, int src, int &total_work,
                     bool print_hop);

int sssp_init(int, int, int *, int *, VALUE_TYPE *) { return -1; }
int sssp_run_adaptive(int, graph_info) { return -1; }
int sssp_cp_data(VALUE_TYPE **) { return -1; }

extern "C" {

// Runs the reference's sssp_sequential exactly as its caller does
// (main.cu:180-193): dist = INT_MAX everywhere, dist[src] = 0, scratch
// prep/hop arrays, then the call.  Returns 0, or -2 on bad arguments,
// -6 when scratch allocation fails.
int ref_sssp_sequential(int n, int nnz, int *row, int *col, int *w, int src, int *dist,
                        long long *total_work) {
    if (n <= 0 || src < 0 || src >= n || !row || !dist) return -2;
    int *prep = (int *)std::malloc(sizeof(int) * (size_t)n);
    int *hop = (int *)std::malloc(sizeof(int) * (size_t)n);
    if (!prep || !hop) {
        std::free(prep);
        std::free(hop);
        return -6;
    }
    for (int i = 0; i < n; i++) dist[i] = INT_MAX;
    dist[src] = 0;
    int work = 0;
    sssp_sequential(n, nnz, row, col, w, dist, prep, hop, src, work, false);
    if (total_work) *total_work = work;
    std::free(prep);
    std::free(hop);
    return 0;
}

}  // extern "C"
