// host_graph.h -- library-private layout of a host CSR graph (mlmq_host_graph),
// shared by the host graph layer (graph_host.cpp) and the device
// preprocessing kernels (reorder.cu).
#pragma once

#include <cstdint>
#include <vector>

struct mlmq_host_graph {
    int n = 0;
    int64_t m = 0;
    std::vector<int> row, col, w, perm;
};
