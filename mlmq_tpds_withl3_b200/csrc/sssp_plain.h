// sssp_plain.h -- host-side entry points of the persistent single-source kernel.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>

namespace mlmq {

struct PlainParams;

// Most threads per CTA of the persistent kernels that keep more than one
// relaxation round in flight (24 worker warps + the manager): their register
// budget is sized for it.
constexpr int PLAIN_MAX_THREADS = 800;
// Register cap of the batched and served kernels: 56 registers fit four CTAs
// of nine warps on an SM (three at the 64-72 registers they would take
// uncapped), and with their counters and per-query parameters in shared
// memory they do not spill at it.
constexpr int SLOT_KERNEL_REGS = 56;

// Dynamic shared memory of one CTA with `workers` worker warps.
size_t plain_smem_bytes(int workers);
// Dynamic shared-memory limit set on every persistent kernel: the largest
// CTA any configuration may launch (31 worker warps).  One limit for all
// solvers, so creating a solver with a smaller CTA never lowers the limit
// below what another live solver launches with.
size_t plain_smem_limit();
// CTAs of the kernel with `unroll` relaxation rounds in flight (1, 2 or 4)
// that fit on one SM (also sets the shared-memory limit).
cudaError_t plain_max_blocks_per_sm(int workers, int unroll, int *blocks);
// Cooperative launch of `grid` CTAs on `stream`.
cudaError_t plain_launch(const PlainParams &p, int unroll, int grid, cudaStream_t stream);

}  // namespace mlmq
