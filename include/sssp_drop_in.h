/*
 * sssp_drop_in.h -- the reference solver's entry points with their original
 * C++ linkage, as exported by libmlmq_b200.so.
 *
 * These replace, one for one, the definitions in the reference's single-GPU
 * solver (hideoze/mlmq_tpds_withl3,
 * evidence/l3_supplement_20260921_v2/single_source/SSSP/sssp_run.cu) that its
 * CLI declares at SS/SSSP/main.cu:15-17:
 *
 *   sssp_init          replaces sssp_run.cu:676  (declared main.cu:15)
 *   sssp_re_init       replaces sssp_run.cu:709
 *   sssp_run_adaptive  replaces sssp_run.cu:888  (declared main.cu:16)
 *   sssp_cp_data       replaces sssp_run.cu:749  (declared main.cu:17)
 *
 * A reference caller needs no header from this library: it keeps its own
 * declarations and links with -lmlmq_b200.  This header is for new C++
 * callers that want the reference's names; it must not be included in the
 * same translation unit as mlmq_b200.h, which declares the same names with C
 * linkage (both sets are exported).
 */
#ifndef MLMQ_SSSP_DROP_IN_H
#define MLMQ_SSSP_DROP_IN_H

#ifndef __cplusplus
#error "sssp_drop_in.h declares C++-linkage symbols; C callers use mlmq_b200.h"
#endif

/* Layout of core/include/graph_info.h:8-22 (the reference's struct; the name
 * is part of sssp_run_adaptive's mangled symbol). */
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

/* RowPtr/ColIdx/edge_data are DEVICE pointers owned by the caller. */
int sssp_init(int m, int nnz, int *RowPtr, int *ColIdx, int *edge_data);
int sssp_re_init();
int sssp_run_adaptive(int src, graph_info info);
/* *node_data_h: malloc()ed host array of m distances; the caller frees it. */
int sssp_cp_data(int **node_data_h);

#endif /* MLMQ_SSSP_DROP_IN_H */
