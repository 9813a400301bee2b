// sssp_plain.cu -- the allocating solver's persistent kernel (interleaved
// {dst, weight} arcs) and its launch helpers.
#include "sssp_plain_body.cuh"
#include "sssp_plain.h"

#include <algorithm>

namespace mlmq {

// K = 32-arc relaxation rounds a warp keeps in flight (mlmq_config.relax_unroll).
// One round needs few registers, so its variant takes CTAs of up to 1024
// threads; the unrolled variants get the register budget of 800 threads.
// kSplit: built with split heavy vertices and the light/heavy split (see
// relax_batch); the variant without them runs graphs that need neither.
template <int K, bool kSplit>
__global__ void __launch_bounds__(K == 1 ? 1024 : PLAIN_MAX_THREADS, 1)
    sssp_plain_kernel(PlainParams p) {
    plain_body<ArcsInterleaved, K, kSplit>(p, blockIdx.x, gridDim.x);
}

namespace {
const void *plain_kernel(int unroll, bool split) {
    switch (unroll) {
        case 1: return split ? (const void *)sssp_plain_kernel<1, true> : (const void *)sssp_plain_kernel<1, false>;
        case 2: return split ? (const void *)sssp_plain_kernel<2, true> : (const void *)sssp_plain_kernel<2, false>;
        default: return split ? (const void *)sssp_plain_kernel<4, true> : (const void *)sssp_plain_kernel<4, false>;
    }
}
// A launch needs the split-capable variant when its graph has pieces or the
// light/heavy split is on.
bool needs_split(const PlainParams &p) { return p.split != nullptr || p.nslots > p.n; }
}  // namespace

// ---- host side ----------------------------------------------------------------

size_t plain_smem_bytes(int workers) { return (size_t)workers * WARP_SMEM_SLOTS * sizeof(uint2); }
size_t plain_smem_limit() { return plain_smem_bytes(31); }

// The smaller of the two variants' occupancies, so that either may be
// launched cooperatively on the grid sized from it.
cudaError_t plain_max_blocks_per_sm(int workers, int unroll, int *blocks) {
    const int threads = 32 * (workers + 1);
    const size_t smem = plain_smem_bytes(workers);
    *blocks = 0;
    for (int split = 0; split < 2; split++) {
        const void *k = plain_kernel(unroll, split != 0);
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)plain_smem_limit());
        if (e != cudaSuccess) return e;
        int b = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k, threads, smem);
        if (e != cudaSuccess) return e;
        *blocks = split ? std::min(*blocks, b) : b;
    }
    return cudaSuccess;
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
    return cudaLaunchKernelExC(&cfg, plain_kernel(unroll, needs_split(p)), args);
}

}  // namespace mlmq
