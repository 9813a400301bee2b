// sssp_plain.cu -- the allocating solver's persistent kernel (interleaved
// {dst, weight} arcs) and its launch helpers.
#include "sssp_plain_body.cuh"
#include "sssp_plain.h"

namespace mlmq {

__global__ void __launch_bounds__(1024, 1) sssp_plain_kernel(PlainParams p) {
    plain_body<ArcsInterleaved>(p, blockIdx.x, gridDim.x);
}

// ---- host side ----------------------------------------------------------------

size_t plain_smem_bytes(int workers) { return (size_t)workers * (L1_CAP + 32) * sizeof(uint2); }

cudaError_t plain_max_blocks_per_sm(int workers, int *blocks) {
    const int threads = 32 * (workers + 1);
    const size_t smem = plain_smem_bytes(workers);
    cudaError_t e = cudaFuncSetAttribute(sssp_plain_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, sssp_plain_kernel, threads, smem);
}

cudaError_t plain_launch(const PlainParams &p, int grid, cudaStream_t stream) {
    const int threads = 32 * (p.workers + 1);
    const size_t smem = plain_smem_bytes(p.workers);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, sssp_plain_kernel, p);
}

}  // namespace mlmq
