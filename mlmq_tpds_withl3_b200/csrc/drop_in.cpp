// drop_in.cpp -- the reference solver's entry points with the reference's own
// C++ linkage, so that its caller (SS/SSSP/main.cu:15-17, which declares
// `extern int sssp_init(...)` etc. without extern "C") links against this
// library unchanged.  Each forwards to the same implementation as the C-linkage
// exports in solver_api.cu.
//
// This translation unit must not see include/mlmq_b200.h: that header declares
// the same names with C linkage.
namespace mlmq {
int dropin_init(int m, int nnz, int *RowPtr, int *ColIdx, int *edge_data);
int dropin_re_init();
int dropin_run(int src);
int dropin_cp_data(int **node_data_h);
}  // namespace mlmq

// Same name and layout as the reference's struct graph_info
// (core/include/graph_info.h:8-22): the name fixes the mangled symbol of
// sssp_run_adaptive, the layout its by-value argument passing.
struct graph_info {
    int m;
    int nnz;
    float avg_nnz;
    float max_nnz;
    float dev_nnz;
    float avg_weight;
    float dev_weight;
    float max_weight;
    float diameter;
};

int sssp_init(int m, int nnz, int *RowPtr, int *ColIdx, int *edge_data) {
    return mlmq::dropin_init(m, nnz, RowPtr, ColIdx, edge_data);
}
int sssp_re_init() { return mlmq::dropin_re_init(); }
int sssp_run_adaptive(int src, graph_info) { return mlmq::dropin_run(src); }
int sssp_cp_data(int **node_data_h) { return mlmq::dropin_cp_data(node_data_h); }
