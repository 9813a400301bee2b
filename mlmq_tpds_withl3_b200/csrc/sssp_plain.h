// sssp_plain.h -- host-side entry points of the persistent single-source kernel.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>

namespace mlmq {

struct PlainParams;

// Dynamic shared memory of one CTA with `workers` worker warps.
size_t plain_smem_bytes(int workers);
// CTAs of the kernel that fit on one SM (also sets the shared-memory limit).
cudaError_t plain_max_blocks_per_sm(int workers, int *blocks);
// Cooperative launch of `grid` CTAs on `stream`.
cudaError_t plain_launch(const PlainParams &p, int grid, cudaStream_t stream);

}  // namespace mlmq
