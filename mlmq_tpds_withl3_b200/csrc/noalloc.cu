// noalloc.cu -- single-source solve that allocates no memory.
//
// Some callers cannot call cudaMalloc while they solve: code running inside a
// framework that owns the device's memory through its own pool allocator,
// an allocation-free real-time or safety-checked path, or a process whose
// device memory was carved up up front.  For them this entry point keeps
// its queue workspace in one file-scope __device__ array that is part of the
// library's device image: it comes into existence when the module loads on
// a device and stays there, on every GPU that loads this library, until the
// process exits.  The caller passes the graph (device CSR) and the output
// distance array; nothing else is allocated, by this code or by a library
// it calls.
//
// Limits and behaviour (also in include/mlmq_b200.h):
//  * workspace: 17 L2 rings of 2^17 slots + one L3 ring of 2^20 slots + one
//    L3 bit per vertex + the control block = MLMQ_NOALLOC_WORKSPACE_BYTES
//    (about 26 MiB);
//  * graphs up to MLMQ_NOALLOC_MAX_VERTICES vertices and MLMQ_NOALLOC_MAX_ARCS
//    arcs, bucket_num <= 16 and at most 8 worker warps per CTA; larger
//    requests are rejected with MLMQ_ERR_RANGE before anything runs;
//  * every call shares the one workspace and leaves its last contents
//    behind; a successful solve leaves every ring slot empty, the kernel
//    clears the counters itself, and after a failed solve the next call
//    clears the rings first.  Calls whose kernels overlap on the GPU (two
//    host threads, or two streams) race on the workspace and corrupt each
//    other: serialise them;
//  * the first call on a device looks the workspace's device address up
//    (cudaGetSymbolAddress, with that device current) and clears it; make
//    that first call before any stream capture on that device.  The set-up
//    is tied to the device's CUDA context: after a cudaDeviceReset the
//    library's device image is loaded again (the array comes back
//    zero-filled, possibly at another address), and the next call repeats
//    the set-up instead of trusting what it found before.
#include "mlmq_b200.h"
#include "solver_internal.h"
#include "sssp_plain.h"
#include "sssp_plain_body.cuh"

#include <cstdio>
#include <mutex>

namespace mlmq {
namespace {

constexpr int NA_RINGS = 17;          // 16 buckets + the urgent ring
constexpr int NA_L2_LOG = 17;
constexpr int NA_L3_LOG = 20;
constexpr int NA_WORKERS = 8;         // keeps in-flight pushes inside half a ring
constexpr size_t NA_CTL_U64 = (ctl::WORDS + 1) / 2 + 32;  // control block, padded
constexpr size_t NA_L2_U64 = (size_t)NA_RINGS << NA_L2_LOG;
constexpr size_t NA_L3_U64 = (size_t)1 << NA_L3_LOG;
constexpr size_t NA_BITS_U64 = (size_t)MLMQ_NOALLOC_MAX_VERTICES / 64;  // L3 vertex bits
constexpr size_t NA_TOTAL_U64 = NA_CTL_U64 + NA_L2_U64 + NA_L3_U64 + NA_BITS_U64;
static_assert(NA_TOTAL_U64 * 8 == MLMQ_NOALLOC_WORKSPACE_BYTES, "header constant out of date");

// The workspace.  Host code must never pass `g_noalloc_ws` itself to a kernel
// or a copy: on the host it names a stand-in, not the device array.  Its
// device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned long long g_noalloc_ws[NA_TOTAL_U64];

// Relaxes one round of 32 arcs at a time (relax_unroll does not apply here).
__global__ void __launch_bounds__(1024, 1) sssp_noalloc_kernel(PlainParams p) {
    plain_body<ArcsSplit, 1>(p, blockIdx.x, gridDim.x);
}

struct DeviceSlot {
    unsigned long long *ws = nullptr;  // device address of g_noalloc_ws
    unsigned long long ctx_id = 0;     // CUDA context the address belongs to (0: unknown)
    bool clean = false;                // every ring slot empty
};
std::mutex g_na_mu;
DeviceSlot g_na_dev[64];

// The current context's unique id (cuCtxGetId, reached through the runtime's
// driver entry points so the library needs no link to the driver library),
// or 0 when it cannot be read.
unsigned long long current_context_id() {
    using GetCurrent = int (*)(void **);
    using GetId = int (*)(void *, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        void *a = nullptr, *b = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault) == cudaSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault) == cudaSuccess) {
            get_current = reinterpret_cast<GetCurrent>(a);
            get_id = reinterpret_cast<GetId>(b);
        }
        cudaGetLastError();
        looked_up = true;
    }
    void *ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
}

// Once per device context, with that device current: resolve the workspace
// address.  A context other than the one the address was found in (the
// device was reset) repeats the set-up and marks the workspace for clearing.
int workspace_for(int dev, DeviceSlot **out) {
    if (dev < 0 || dev >= 64) return MLMQ_ERR_NODEV;
    DeviceSlot &d = g_na_dev[dev];
    const unsigned long long ctx = current_context_id();
    if (!d.ws || ctx == 0 || ctx != d.ctx_id) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_ws);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_ws)");
        d.ws = static_cast<unsigned long long *>(ptr);
        d.ctx_id = ctx;
        d.clean = false;
    }
    *out = &d;
    return MLMQ_OK;
}

}  // namespace
}  // namespace mlmq

using namespace mlmq;

extern "C" int mlmq_sssp_solve_noalloc(int n, int m, const int *d_row, const int *d_col,
                                       const int *d_w, int src, int *d_dist,
                                       const mlmq_config *cfg_in, void *stream) {
    if (n <= 0 || m < 0 || !d_row || !d_dist || (m > 0 && (!d_col || !d_w)) || src < 0 ||
        src >= n)
        return MLMQ_ERR_ARG;
    if (n > MLMQ_NOALLOC_MAX_VERTICES || m > MLMQ_NOALLOC_MAX_ARCS) {
        std::fprintf(stderr,
                     "mlmq_sssp_solve_noalloc: graph of %d vertices / %d arcs exceeds the "
                     "fixed workspace (at most %d vertices, %d arcs); use mlmq_solver_*\n",
                     n, m, MLMQ_NOALLOC_MAX_VERTICES, MLMQ_NOALLOC_MAX_ARCS);
        return MLMQ_ERR_RANGE;
    }
    mlmq_config cfg;
    int rc = MLMQ_OK;
    if (cfg_in) cfg = *cfg_in;
    else if ((rc = mlmq_config_default(&cfg))) return rc;
    if ((rc = validate_config(cfg))) return rc;
    if (cfg.bucket_num > NA_RINGS - 1) {
        std::fprintf(stderr, "mlmq_sssp_solve_noalloc: bucket_num %d > %d (fixed workspace)\n",
                     cfg.bucket_num, NA_RINGS - 1);
        return MLMQ_ERR_RANGE;
    }
    const int workers = cfg.warps_per_block < NA_WORKERS ? cfg.warps_per_block : NA_WORKERS;

    int dev = 0, sms = 0;
    if ((rc = cuda_fail(cudaGetDevice(&dev), "cudaGetDevice"))) return rc;
    if ((rc = device_sm_count(&sms))) return rc;
    cudaStream_t st = (cudaStream_t)stream;

    std::lock_guard<std::mutex> lk(g_na_mu);
    DeviceSlot *slot = nullptr;
    if ((rc = workspace_for(dev, &slot))) return rc;
    unsigned long long *ctl_base = slot->ws;
    unsigned long long *l2 = ctl_base + NA_CTL_U64;
    unsigned long long *l3 = l2 + NA_L2_U64;
    unsigned *l3bits = reinterpret_cast<unsigned *>(l3 + NA_L3_U64);  // cleared by the kernel
    if (!slot->clean) {
        rc = cuda_fail(cudaMemsetAsync(ctl_base, 0, NA_CTL_U64 * 8, st), "clear control");
        if (!rc) rc = cuda_fail(cudaMemsetAsync(l2, 0xff, (NA_L2_U64 + NA_L3_U64) * 8, st),
                                "clear rings");
        if (rc) return rc;
    }

    int bps = 0;
    const int threads = 32 * (workers + 1);
    const size_t smem = plain_smem_bytes(workers);
    rc = cuda_fail(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, sssp_noalloc_kernel,
                                                                 threads, smem), "occupancy");
    if (rc) return rc;
    if (bps < 1) return MLMQ_ERR_UNSUPPORTED;
    int grid = cfg.work_blocks > 0 ? cfg.work_blocks : sms;
    if (grid > bps * sms) grid = bps * sms;

    PlainParams p{};
    p.n = n;
    p.nslots = n;  // the caller's CSR has no split pieces
    p.nids = n;
    p.row = d_row;
    p.arcs = nullptr;
    p.tiles = nullptr;  // the caller's CSR is read in place
    p.tile_stride = 2;
    p.col = d_col;
    p.w = d_w;
    p.dist = d_dist;
    p.src = src;
    p.l2 = l2;
    p.l3 = l3;
    p.l3bits = l3bits;
    p.ctlw = reinterpret_cast<unsigned *>(ctl_base);
    p.nb = cfg.bucket_num;
    p.bm = cfg.bucket_max;
    p.batch = cfg.l2_batch;
    p.min_read = cfg.min_read;
    p.large = cfg.large_degree;
    p.l1_spill = cfg.l1_spill;
    p.l1_vector = cfg.queue_type == MLMQ_L1V_L2DQ;
    p.l1_keep = cfg.l1_keep;
    p.l1_ahead = cfg.l1_ahead;
    p.topup = cfg.topup;
    p.bucket_sync = cfg.bucket_sync;
    p.split = nullptr;  // the light/heavy split needs vertex tiles
    p.precheck = cfg.relax_precheck;
    p.delta = (unsigned)cfg.delta;
    p.l2_log = NA_L2_LOG;
    p.l3_log = NA_L3_LOG;
    p.workers = workers;
    p.timeout_ns = (unsigned long long)cfg.timeout_ms * 1000000ull;

    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3((unsigned)grid);
    lc.blockDim = dim3((unsigned)threads);
    lc.dynamicSmemBytes = smem;
    lc.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    slot->clean = false;
    rc = cuda_fail(cudaLaunchKernelEx(&lc, sssp_noalloc_kernel, p), "no-alloc launch");
    if (rc) return rc;
    unsigned status = 0;
    rc = cuda_fail(cudaMemcpyAsync(&status, p.ctlw + ctl::STATUS, sizeof(status),
                                   cudaMemcpyDeviceToHost, st), "status copy");
    if (!rc) rc = cuda_fail(cudaStreamSynchronize(st), "no-alloc solve");
    if (rc) return rc;
    rc = status_to_error(status);
    // A finished solve consumed every record it reserved: the rings are empty.
    slot->clean = (status & ST_DONE) && !(status & (ST_TIMEOUT | ST_QUEUE_FULL));
    return rc;
}
