// oracle/ref_chain.cpp -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// Puts a C entry point in front of the reference's own chain-shortcut builder,
// `l3_chain_shortcut_view::build` from SSSP/l3/l3_chain_shortcuts.h:23-109,
// which oracle/Makefile compiles unchanged from the reference tree.  Tests load
// the result with ctypes and compare the product's mlmq_hgraph_chain_shortcuts
// with it arc for arc.
#include <cstdint>
#include <cstring>
#include <exception>

#include "l3_chain_shortcuts.h"

extern "C" {

// Builds G+ for (n, m, row, dst, w) with the given cut and source.  On success
// writes rows (n + 1 entries) and up to `cap` arcs into out_dst/out_w, the arc
// count into *out_m and the builder's counters into stats[5] (eligible
// vertices, shortcuts, longest path, overflow paths, represented edges).
// Returns 0, -2 when the builder threw, -8 when `cap` is too small.
int ref_chain_shortcuts(int n, int m, const int *row, const int *dst, const int *w, int cut,
                        int source, int *out_row, int *out_dst, int *out_w, long long cap,
                        long long *out_m, long long *stats) {
    l3_chain_shortcut_view v;
    try {
        v.build(n, m, row, dst, w, cut, source);
    } catch (const std::exception &) {
        return -2;
    }
    const long long mm = (long long)v.destinations.size();
    if (mm > cap) return -8;
    std::memcpy(out_row, v.rows.data(), sizeof(int) * ((size_t)n + 1));
    std::memcpy(out_dst, v.destinations.data(), sizeof(int) * (size_t)mm);
    std::memcpy(out_w, v.weights.data(), sizeof(int) * (size_t)mm);
    *out_m = mm;
    stats[0] = v.eligible_vertices;
    stats[1] = v.shortcuts;
    stats[2] = v.longest_path;
    stats[3] = v.overflow_paths;
    stats[4] = v.represented_edges;
    return 0;
}

}  // extern "C"
