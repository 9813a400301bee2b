// sssp_plain.cu -- the allocating solver's persistent kernel (interleaved
// {dst, weight} arcs) and its launch helpers.
#include "sssp_plain_body.cuh"
#include "sssp_plain.h"

namespace mlmq {

// K = 32-arc relaxation rounds a warp keeps in flight (mlmq_config.relax_unroll).
// One round needs few registers, so its variant takes CTAs of up to 1024
// threads; the unrolled variants get the register budget of 800 threads.
template <int K>
__global__ void __launch_bounds__(K == 1 ? 1024 : PLAIN_MAX_THREADS, 1)
    sssp_plain_kernel(PlainParams p) {
    plain_body<ArcsInterleaved, K>(p, blockIdx.x, gridDim.x);
}

namespace {
const void *plain_kernel(int unroll) {
    switch (unroll) {
        case 1: return (const void *)sssp_plain_kernel<1>;
        case 2: return (const void *)sssp_plain_kernel<2>;
        default: return (const void *)sssp_plain_kernel<4>;
    }
}
}  // namespace

// ---- host side ----------------------------------------------------------------

size_t plain_smem_bytes(int workers) { return (size_t)workers * WARP_SMEM_SLOTS * sizeof(uint2); }
size_t plain_smem_limit() { return plain_smem_bytes(31); }

cudaError_t plain_max_blocks_per_sm(int workers, int unroll, int *blocks) {
    const int threads = 32 * (workers + 1);
    const size_t smem = plain_smem_bytes(workers);
    const void *k = plain_kernel(unroll);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)plain_smem_limit());
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, k, threads, smem);
}

cudaError_t plain_launch(const PlainParams &p, int unroll, int grid, cudaStream_t stream) {
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
    void *args[] = {const_cast<PlainParams *>(&p)};
    return cudaLaunchKernelExC(&cfg, plain_kernel(unroll), args);
}

}  // namespace mlmq
