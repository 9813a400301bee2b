// sssp_server.cu -- continuous-batching query server: one persistent launch
// that keeps serving single-source queries on HBM-resident graphs while new
// queries arrive.
//
// The grid is split into `slots` contiguous CTA groups (as in the batched
// launch).  Each slot owns a distance buffer, queue rings and a control
// block.  The host hands a query to a free slot by copying a command into
// the slot's mailbox in device memory (two small host-to-device copies on
// their own stream: the fields, then the sequence number); the slot's first
// CTA polls the mailbox, publishes the command to the rest of its group, and
// the group runs the single-source algorithm (sssp_plain_body.cuh).  Idle
// slots therefore poll HBM, not host memory: host-memory polling by dozens
// of idle slots loaded PCIe enough to delay the result copies by ~200 ms,
// which kept slots idle longer -- a feedback loop that held a 64-slot
// server near 230 queries/s.  At the
// end a group barrier makes sure every CTA of the slot has left the solve,
// and the first CTA writes the completion (sequence number, status, counters)
// into mapped host memory.  The host copies the distances out on another
// stream while the server keeps running; the slot takes its next query once
// that copy is done.  Queries on different graphs and of different sizes run
// side by side; a query's result does not depend on what else runs.
//
// Every wait is bounded.  An idle slot waits for its next command until the
// server's lifetime ends or the host sets the shutdown flag.  Everything a
// slot does for one query -- the solve and the group barriers around its
// end -- is bounded by that query's own time limit plus a margin, so a query
// always gets a completion within that time: a slot whose CTAs cannot all
// meet reports ST_TIMEOUT | ST_SLOT_LOST and takes no further queries.
#include "mlmq_b200.h"
#include "solver_internal.h"
#include "sssp_plain.h"
// Per-warp counters in shared memory (see mlmq_queue.cuh).
#define MLMQ_WARP_STATS_SMEM 1
#include "sssp_plain_body.cuh"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <vector>

namespace mlmq {
namespace {

constexpr int SRV_CTL_STRIDE = 512;  // words per slot control block
// Words of the slot control block used by the server around a solve (the
// solve itself uses words below ctl::WORDS).
constexpr int SRV_CMD = 456;      // device copy of the command: row, arcs, tiles (2 words each),
                                  // n, src, delta, topup, l1_ahead, bucket_max, nslots,
                                  // bucket_sync, nids, split (2 words)
constexpr int SRV_GO = 480;       // published command sequence (device)
constexpr int SRV_STOP = 481;     // shutdown seen by the slot leader
constexpr int SRV_LOST = 482;     // a CTA of the slot gave up on a group barrier
constexpr int SRV_DIGEST = 484;   // u64: digest of the slot's last result (8-byte aligned)
constexpr int SRV_BAR_COUNT = 488;
constexpr int SRV_BAR_GEN = 489;
// Time the CTAs of a slot may take, past the query's own limit, to meet
// after a solve (every CTA leaves the solve by that limit); the environment
// variable MLMQ_SERVER_MEET_MS overrides it at server creation.
constexpr unsigned long long SRV_MEET_NS = 2000000000ull;

__device__ __forceinline__ unsigned long long ld_acquire64(const volatile unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Command, one per slot: staged in pinned host memory, copied into the
// slot's device mailbox -- every field first, then `seq` (a second copy in
// the same stream, so the fields are in device memory before it lands).
struct alignas(64) SlotCommand {
    volatile unsigned long long seq;
    const int *row;
    const int2 *arcs;
    const int4 *tiles;
    int n;
    int src;
    int nslots, nids;
    // per-query settings (the server's configuration unless overridden)
    unsigned delta;
    int topup, l1_ahead, bm, bucket_sync;
    const int *split;
};
// Host-mapped completion, one per slot, written by the device.
struct alignas(64) SlotCompletion {
    volatile unsigned long long seq;
    volatile unsigned status;
    volatile unsigned first_max;
    volatile unsigned long long relaxed, pushed;
    // device clock (ns): the slot took the command / reported the result
    volatile unsigned long long t_start, t_end;
    volatile unsigned lost;  // 1: the slot's CTAs stopped serving (see SRV_LOST)
    volatile unsigned long long digest;  // digest_term sum over the result's vertices
};

struct ServerParams {
    PlainParams base;             // queue configuration shared by all slots
    SlotCommand *cmd;             // device mailboxes, [slots]
    SlotCompletion *done;         // mapped, [slots]
    volatile unsigned *shutdown;  // device
    int *dist;                    // slots * max_n
    unsigned long long *l2, *l3;
    unsigned *l3bits;             // slots * bits_words
    size_t bits_words;
    unsigned *ctl;                // slots * SRV_CTL_STRIDE
    const int *cta_slot;          // [grid] slot of each CTA
    const int *slot_first;        // [slots + 1] first CTA of each slot
    int slots, max_n;
    unsigned long long lifetime_ns;
    unsigned long long meet_ns;  // how long past a query's limit its CTAs may take to meet
    int absent_cta;  // test of the bounded barrier: this CTA leaves after its first solve (-1: none)
};

// Group barrier on words outside the solve's control words.  A CTA that
// gives up at `deadline` marks the slot lost (SRV_LOST); a CTA that passes
// the barrier but finds the mark set fails too, so the CTAs of a slot agree
// that it is lost unless one gave up after the others had checked -- then
// the next command finds the mark (see the command wait).
__device__ bool group_barrier(unsigned *c, unsigned gsize, unsigned long long deadline) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        unsigned gen = ld_acquire(c + SRV_BAR_GEN);
        __threadfence();
        if (atomicAdd(c + SRV_BAR_COUNT, 1u) == gsize - 1) {
            st_relaxed(c + SRV_BAR_COUNT, 0u);
            __threadfence();
            st_release(c + SRV_BAR_GEN, gen + 1);
        } else {
            unsigned ns = 64;
            while (ld_acquire(c + SRV_BAR_GEN) == gen) {
                if (globaltimer() > deadline) {
                    atomicOr(c + SRV_LOST, 1u);
                    ok = 0;
                    break;
                }
                __nanosleep(ns);
                if (ns < 2048) ns <<= 1;
            }
        }
        if (ok && ld_acquire(c + SRV_LOST)) ok = 0;
    }
    __syncthreads();
    return ok != 0;
}

template <int K>
__global__ void __maxnreg__(SLOT_KERNEL_REGS) sssp_server_kernel(ServerParams sp) {
    // Slot s is the CTA group [slot_first[s], slot_first[s + 1]); slots may
    // differ in size (small ones for latency-bound queries, wide ones for
    // throughput-bound queries).
    // The slot's identity and the loop's state live in shared memory, not in
    // registers that would stay allocated through every solve.
    struct SlotState {
        unsigned long long end, seen, t_go;
        unsigned *c;
        unsigned s, grank, gsize;
    };
    __shared__ SlotState ss;
    __shared__ unsigned long long go_seq, go_time;
    __shared__ int stop;
    if (threadIdx.x == 0) {
        const unsigned s = (unsigned)sp.cta_slot[blockIdx.x];
        const unsigned lo = (unsigned)sp.slot_first[s];
        const unsigned hi = (unsigned)sp.slot_first[s + 1];
        ss.s = s;
        ss.grank = blockIdx.x - lo;
        ss.gsize = hi - lo;
        ss.c = sp.ctl + (size_t)s * SRV_CTL_STRIDE;
        ss.end = globaltimer() + sp.lifetime_ns;
        ss.seen = 0;
    }
    __syncthreads();
    for (;;) {
        // ---- wait for the slot's next command ------------------------------
        if (threadIdx.x == 0) {
            const unsigned s = ss.s, grank = ss.grank;
            unsigned *c = ss.c;
            const unsigned long long end = ss.end, seen = ss.seen;
            stop = 0;
            unsigned ns = 256;
            for (;;) {
                if (ld_acquire(c + SRV_LOST)) {
                    // A CTA of this slot gave up on a barrier after the last
                    // completion: the slot can no longer meet; tell the host.
                    if (grank == 0) {
                        sp.done[s].lost = 1u;
                        __threadfence_system();
                    }
                    stop = 1;
                    break;
                }
                if (grank == 0) {
                    if (ld_acquire(const_cast<const unsigned *>(sp.shutdown))) {
                        st_release(c + SRV_STOP, 1u);
                        stop = 1;
                        break;
                    }
                    const unsigned long long q = ld_acquire64(&sp.cmd[s].seq);
                    if (q != seen) {
                        go_seq = q;
                        go_time = globaltimer();
                        // Copy the command into the control block for the group.
                        const volatile SlotCommand &cm = sp.cmd[s];
                        const unsigned long long row = (unsigned long long)cm.row;
                        const unsigned long long arcs = (unsigned long long)cm.arcs;
                        c[SRV_CMD + 0] = (unsigned)row;
                        c[SRV_CMD + 1] = (unsigned)(row >> 32);
                        c[SRV_CMD + 2] = (unsigned)arcs;
                        c[SRV_CMD + 3] = (unsigned)(arcs >> 32);
                        c[SRV_CMD + 4] = (unsigned)cm.n;
                        c[SRV_CMD + 5] = (unsigned)cm.src;
                        const unsigned long long tiles = (unsigned long long)cm.tiles;
                        c[SRV_CMD + 6] = (unsigned)tiles;
                        c[SRV_CMD + 7] = (unsigned)(tiles >> 32);
                        c[SRV_CMD + 8] = cm.delta;
                        c[SRV_CMD + 9] = (unsigned)cm.topup;
                        c[SRV_CMD + 10] = (unsigned)cm.l1_ahead;
                        c[SRV_CMD + 11] = (unsigned)cm.bm;
                        c[SRV_CMD + 12] = (unsigned)cm.nslots;
                        c[SRV_CMD + 13] = (unsigned)cm.bucket_sync;
                        c[SRV_CMD + 14] = (unsigned)cm.nids;
                        const unsigned long long spl = (unsigned long long)cm.split;
                        c[SRV_CMD + 15] = (unsigned)spl;
                        c[SRV_CMD + 16] = (unsigned)(spl >> 32);
                        *reinterpret_cast<unsigned long long *>(c + SRV_DIGEST) = 0ull;
                        __threadfence();
                        // publish the sequence number (low 32 bits) to the group
                        st_release(c + SRV_GO, (unsigned)q);
                        break;
                    }
                } else {
                    if (ld_acquire(c + SRV_STOP)) {
                        stop = 1;
                        break;
                    }
                    const unsigned q = ld_acquire(c + SRV_GO);
                    if (q != (unsigned)seen) {
                        go_seq = seen + (unsigned)(q - (unsigned)seen);
                        break;
                    }
                }
                if (globaltimer() > end) {
                    stop = 1;
                    break;
                }
                __nanosleep(ns);
                if (ns < 4096) ns <<= 1;
            }
        }
        __syncthreads();
        if (stop) return;
        // ---- one solve --------------------------------------------------------
        // The query's parameters go to shared memory, not registers (as in
        // the batched kernel).  Every thread has passed the __syncthreads
        // above since the last read of the previous query's copy.
        __shared__ PlainParams cta_params;
        if (threadIdx.x == 0) {
            const unsigned s = ss.s;
            unsigned *c = ss.c;
            ss.seen = go_seq;
            // This CTA's view of when the query started: its solve ends by
            // this plus the query's time limit.
            ss.t_go = globaltimer();
            PlainParams p = sp.base;
            const volatile unsigned *cmd = c + SRV_CMD;
            p.row = (const int *)(((unsigned long long)cmd[1] << 32) | cmd[0]);
            p.arcs = (const int2 *)(((unsigned long long)cmd[3] << 32) | cmd[2]);
            p.tiles = (const int4 *)(((unsigned long long)cmd[7] << 32) | cmd[6]);
            p.delta = cmd[8];
            p.topup = (int)cmd[9];
            p.l1_ahead = (int)cmd[10];
            p.bm = (int)cmd[11];
            p.nslots = (int)cmd[12];
            p.bucket_sync = (int)cmd[13];
            p.nids = (int)cmd[14];
            p.split = (const int *)(((unsigned long long)cmd[16] << 32) | cmd[15]);
            p.n = (int)cmd[4];
            p.src = (int)cmd[5];
            p.dist = sp.dist + (size_t)s * sp.max_n;
            p.l2 = sp.l2 + ((size_t)s * (p.nb + 1) << p.l2_log);
            p.l3 = sp.l3 + ((size_t)s << p.l3_log);
            p.l3bits = sp.l3bits + (size_t)s * sp.bits_words;
            p.ctlw = c;
            cta_params = p;
        }
        __syncthreads();
        const PlainParams &p = cta_params;
        plain_body<ArcsInterleaved, K>(p, ss.grank, ss.gsize);
        const unsigned s = ss.s, grank = ss.grank, gsize = ss.gsize;
        unsigned *c = ss.c;
        if ((int)blockIdx.x == sp.absent_cta) return;  // test: a CTA that never arrives
        // Every CTA of the slot leaves the solve before anything else: after
        // this barrier nothing writes the status word any more, so every CTA
        // reads the same final status (read before it, a CTA could miss a
        // bit that a slower CTA still sets, and the CTAs would then take
        // different barriers below).  Bounded by the query's own limit.
        bool ok = group_barrier(c, gsize, ss.t_go + p.timeout_ns + sp.meet_ns);
        __shared__ unsigned solve_status;
        if (threadIdx.x == 0) solve_status = ld_acquire(c + ctl::STATUS);
        __syncthreads();
        if (ok && (solve_status & (ST_TIMEOUT | ST_QUEUE_FULL))) {
            // A solve that stopped early leaves records in the rings: the
            // group empties them before the slot is reused.
            const size_t l2n = (size_t)(p.nb + 1) << p.l2_log, l3n = (size_t)1 << p.l3_log;
            for (size_t i = (size_t)grank * blockDim.x + threadIdx.x; i < l2n + l3n;
                 i += (size_t)gsize * blockDim.x) {
                if (i < l2n) p.l2[i] = SENT;
                else p.l3[i - l2n] = SENT;
            }
        }
        if (ok) {
            // Digest of the result, one pass over the distances by the whole
            // group; the host compares it with a reference digest without
            // holding every result (mlmq_server_poll_results).
            __shared__ unsigned long long cta_sum;
            if (threadIdx.x == 0) cta_sum = 0ull;
            __syncthreads();
            unsigned long long part = 0ull;
            for (size_t i = (size_t)grank * blockDim.x + threadIdx.x; i < (size_t)p.n;
                 i += (size_t)gsize * blockDim.x)
                part += digest_term(i, __ldcg(p.dist + i));
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(FULL, part, o);
            if ((threadIdx.x & 31) == 0) atomicAdd(&cta_sum, part);
            __syncthreads();
            if (threadIdx.x == 0)
                atomicAdd(reinterpret_cast<unsigned long long *>(c + SRV_DIGEST), cta_sum);
            ok = group_barrier(c, gsize, globaltimer() + sp.meet_ns);
        }
        if (grank == 0 && threadIdx.x == 0) {
            const unsigned long long *u = reinterpret_cast<const unsigned long long *>(c + ctl::STATS);
            unsigned st = solve_status;
            // A grid barrier of the solve that gave up left its arrival count
            // behind; no CTA of the slot is inside the solve now.
            if (st & ST_TIMEOUT) st_relaxed(c + ctl::BAR_COUNT, 0u);
            if (!ok) {
                st |= ST_TIMEOUT | ST_SLOT_LOST;
                sp.done[s].lost = 1u;
            }
            sp.done[s].status = st;
            sp.done[s].digest = ld_relaxed64(reinterpret_cast<const unsigned long long *>(c + SRV_DIGEST));
            sp.done[s].first_max = (unsigned)u[ctl::ST_FIRST_MAX];
            sp.done[s].relaxed = u[ctl::ST_RELAXED];
            sp.done[s].pushed = u[ctl::ST_PUSHED];
            sp.done[s].t_start = go_time;
            sp.done[s].t_end = globaltimer();
            __threadfence_system();
            sp.done[s].seq = ss.seen;
            __threadfence_system();
        }
        if (!ok) return;
    }
}

const void *server_kernel(int unroll) {
    switch (unroll) {
        case 1: return (const void *)sssp_server_kernel<1>;
        case 2: return (const void *)sssp_server_kernel<2>;
        default: return (const void *)sssp_server_kernel<4>;
    }
}

}  // namespace
}  // namespace mlmq

using namespace mlmq;

struct mlmq_server {
    int device = 0;
    mlmq_config cfg{};
    int slots = 0, max_n = 0, grid = 0, workers = 0, l2_log = 0, l3_log = 0;
    int *d_dist = nullptr;
    unsigned long long *d_l2 = nullptr, *d_l3 = nullptr;
    unsigned *d_l3bits = nullptr;
    size_t bits_words = 0;
    unsigned *d_ctl = nullptr;
    int *d_cta_slot = nullptr, *d_slot_first = nullptr;
    std::vector<int> slot_ctas;   // CTAs of each slot
    SlotCommand *h_cmd = nullptr;   // pinned staging of each slot's command
    SlotCommand *d_cmd = nullptr;   // device mailboxes
    SlotCompletion *h_done = nullptr;
    unsigned *h_shutdown = nullptr; // pinned staging of the shutdown flag
    unsigned *d_shutdown = nullptr;
    cudaStream_t kstream = nullptr, cstream = nullptr;
    cudaStream_t qstream = nullptr;  // command and shutdown copies
    cudaEvent_t kdone = nullptr;
    bool running = false;
    std::mutex mu;
    struct Slot {
        unsigned long long seq = 0;     // last command issued
        bool busy = false;              // solving or copying out
        bool copying = false;
        bool lost = false;              // the slot's CTAs stopped serving
        const mlmq_graph *g = nullptr;  // graph of the query in the slot (one reference)
        unsigned long long ticket = 0;
        int *h_out = nullptr;
        int n = 0;
        cudaEvent_t copied = nullptr;
        unsigned status = 0;
        unsigned long long relaxed = 0;
        unsigned long long solve_ns = 0;
        unsigned long long digest = 0;
    };
    std::vector<Slot> st;
    unsigned long long next_ticket = 1;
    struct Finished {
        unsigned long long ticket;
        int status;
        unsigned long long solve_ns;  // device time from command pickup to result
        unsigned long long digest;    // device digest of the distances (0 when none)
    };
    std::deque<Finished> finished;
};

namespace {

// `layout` (CTAs per slot, `slots` entries) or null for an even split of the
// largest co-resident grid into at most `slots` slots (fewer when device
// memory runs short).
int server_create(int slots, const int *layout, int max_vertices, const mlmq_config *cfg_in,
                  int lifetime_ms, mlmq_server **out) {
    if (!out || slots < 1 || max_vertices < 1 || lifetime_ms < 1) return MLMQ_ERR_ARG;
    if (layout)
        for (int s = 0; s < slots; s++)
            if (layout[s] < 1) return MLMQ_ERR_ARG;
    mlmq_config cfg;
    int rc = MLMQ_OK;
    if (cfg_in) cfg = *cfg_in;
    else {
        if ((rc = mlmq_config_default(&cfg))) return rc;
        cfg.warps_per_block = 8;
    }
    if ((rc = validate_config(cfg))) return rc;
    if (cfg.warps_per_block > MLMQ_MAX_UNROLLED_WARPS) return MLMQ_ERR_ARG;
    int sms = 0;
    if ((rc = device_sm_count(&sms))) return rc;
    auto *sv = new (std::nothrow) mlmq_server;
    if (!sv) return MLMQ_ERR_NOMEM;
    sv->cfg = cfg;
    sv->workers = cfg.warps_per_block;
    sv->l2_log = cfg.l2_cap_log2 ? cfg.l2_cap_log2 : MLMQ_MIN_RING_LOG2;
    sv->l3_log = cfg.l3_cap_log2 ? cfg.l3_cap_log2 : l3_ring_log2(max_vertices, max_vertices);
    sv->bits_words = l3_bits_bytes(max_vertices) / sizeof(unsigned);
    sv->max_n = max_vertices;
    rc = cuda_fail(cudaGetDevice(&sv->device), "cudaGetDevice");
    // Admission by free device memory: as many slots as fit after a reserve.
    const size_t per_slot = sizeof(int) * (size_t)max_vertices +
                            8 * (((size_t)(cfg.bucket_num + 1) << sv->l2_log) + ((size_t)1 << sv->l3_log)) +
                            4 * SRV_CTL_STRIDE + 4 * sv->bits_words;
    size_t free_b = 0, total_b = 0;
    // Memory the library's pool keeps for reuse counts as free here.
    if (!rc) rc = mlmq_release_cached();
    if (!rc) rc = cuda_fail(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    if (!rc) {
        const size_t reserve = (size_t)2 << 30;
        const size_t fit = free_b > reserve ? (free_b - reserve) / per_slot : 0;
        sv->slots = (int)std::min<size_t>((size_t)slots, fit);
        if (sv->slots < 1 || (layout && sv->slots < slots)) rc = MLMQ_ERR_NOMEM;
    }
    int bps = 0;
    const int threads = 32 * (sv->workers + 1);
    const size_t smem = plain_smem_bytes(sv->workers);
    const void *kern = server_kernel(cfg.relax_unroll);
    if (!rc) rc = cuda_fail(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)plain_smem_limit()), "server smem");
    if (!rc) rc = cuda_fail(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, threads, smem),
                            "server occupancy");
    if (!rc && layout) {
        long long total = 0;
        for (int s = 0; s < slots; s++) total += layout[s];
        if (total > (long long)bps * sms) {
            std::fprintf(stderr, "mlmq_server_create_layout: %lld CTAs requested, %d fit\n", total,
                         bps * sms);
            rc = MLMQ_ERR_RANGE;
        } else {
            sv->grid = (int)total;
            sv->slot_ctas.assign(layout, layout + slots);
        }
    } else if (!rc) {
        sv->grid = cfg.work_blocks > 0 ? std::min(cfg.work_blocks, bps * sms) : bps * sms;
        sv->slots = std::min(sv->slots, sv->grid);
        const long long g = sv->grid, n = sv->slots;
        for (long long s = 0; s < n; s++)
            sv->slot_ctas.push_back((int)(((s + 1) * g + n - 1) / n - (s * g + n - 1) / n));
    }
    const size_t ns = (size_t)sv->slots;
    std::vector<int> cta_slot, slot_first(1, 0);
    for (int s = 0; s < (int)sv->slot_ctas.size(); s++) {
        for (int c = 0; c < sv->slot_ctas[s]; c++) cta_slot.push_back(s);
        slot_first.push_back(slot_first.back() + sv->slot_ctas[s]);
    }
    // Device memory from the stream-ordered pool, host memory from the
    // pinned pool: destroying a server never synchronises the device (a
    // plain cudaFree would wait for every other running kernel).
    if (!rc) rc = cuda_fail(cudaStreamCreateWithFlags(&sv->kstream, cudaStreamNonBlocking), "kstream");
    if (!rc) rc = cuda_fail(cudaStreamCreateWithFlags(&sv->cstream, cudaStreamNonBlocking), "cstream");
    if (!rc) rc = cuda_fail(cudaStreamCreateWithFlags(&sv->qstream, cudaStreamNonBlocking), "qstream");
    cudaStream_t ks = sv->kstream;
    if (!rc) rc = dev_alloc(&sv->d_cta_slot, sizeof(int) * cta_slot.size(), ks, "server CTA map");
    if (!rc) rc = dev_alloc(&sv->d_slot_first, sizeof(int) * slot_first.size(), ks, "server slots");
    if (!rc) rc = cuda_fail(cudaMemcpyAsync(sv->d_cta_slot, cta_slot.data(), sizeof(int) * cta_slot.size(),
                                            cudaMemcpyHostToDevice, ks), "H2D CTA map");
    if (!rc) rc = cuda_fail(cudaMemcpyAsync(sv->d_slot_first, slot_first.data(),
                                            sizeof(int) * slot_first.size(), cudaMemcpyHostToDevice, ks),
                            "H2D slots");
    if (!rc) rc = dev_alloc(&sv->d_dist, sizeof(int) * ns * (size_t)max_vertices, ks, "server dist");
    if (!rc) rc = dev_alloc(&sv->d_l2, 8 * ns * ((size_t)(cfg.bucket_num + 1) << sv->l2_log), ks, "server L2");
    if (!rc) rc = dev_alloc(&sv->d_l3, 8 * (ns << sv->l3_log), ks, "server L3");
    if (!rc) rc = dev_alloc(&sv->d_l3bits, 4 * ns * sv->bits_words, ks, "server L3 bits");
    if (!rc) rc = dev_alloc(&sv->d_ctl, 4 * ns * SRV_CTL_STRIDE, ks, "server ctl");
    if (!rc) rc = pinned_alloc(&sv->h_cmd, sizeof(SlotCommand) * ns);
    if (!rc) rc = dev_alloc(&sv->d_cmd, sizeof(SlotCommand) * ns, ks, "server mailboxes");
    if (!rc) rc = dev_alloc(&sv->d_shutdown, 64, ks, "server shutdown flag");
    if (!rc) rc = pinned_alloc(&sv->h_done, sizeof(SlotCompletion) * ns);
    if (!rc) rc = pinned_alloc(&sv->h_shutdown, 64);
    if (!rc) rc = cuda_fail(cudaEventCreateWithFlags(&sv->kdone, cudaEventDisableTiming), "kdone");
    if (!rc) {
        std::memset((void *)sv->h_cmd, 0, sizeof(SlotCommand) * ns);
        std::memset((void *)sv->h_done, 0, sizeof(SlotCompletion) * ns);
        *sv->h_shutdown = 0;
        sv->st.resize(ns);
        for (auto &sl : sv->st)
            if (!rc) rc = cuda_fail(cudaEventCreateWithFlags(&sl.copied, cudaEventDisableTiming), "copy event");
    }
    if (!rc) rc = cuda_fail(cudaMemsetAsync(sv->d_l2, 0xff, 8 * ns * ((size_t)(cfg.bucket_num + 1) << sv->l2_log), sv->kstream), "reset L2");
    if (!rc) rc = cuda_fail(cudaMemsetAsync(sv->d_l3, 0xff, 8 * (ns << sv->l3_log), sv->kstream), "reset L3");
    if (!rc) rc = cuda_fail(cudaMemsetAsync(sv->d_ctl, 0, 4 * ns * SRV_CTL_STRIDE, sv->kstream), "reset ctl");
    if (!rc) rc = cuda_fail(cudaMemsetAsync(sv->d_cmd, 0, sizeof(SlotCommand) * ns, sv->kstream), "reset mailboxes");
    if (!rc) rc = cuda_fail(cudaMemsetAsync(sv->d_shutdown, 0, 64, sv->kstream), "reset shutdown");
    if (!rc) {
        ServerParams sp{};
        PlainParams &b = sp.base;
        b.nb = cfg.bucket_num;
        b.bm = cfg.bucket_max;
        b.batch = cfg.l2_batch;
        b.min_read = cfg.min_read;
        b.large = cfg.large_degree;
        b.l1_spill = cfg.l1_spill;
        b.l1_vector = cfg.queue_type == MLMQ_L1V_L2DQ;
        b.l1_keep = cfg.l1_keep;
        b.l1_ahead = cfg.l1_ahead;
        b.topup = cfg.topup;
        b.bucket_sync = cfg.bucket_sync;
        b.tile_stride = cfg.vertex_tiles == 2 ? 4 : 2;
        b.split = nullptr;  // per query
        b.precheck = cfg.relax_precheck;
        b.delta = (unsigned)cfg.delta;
        b.l2_log = sv->l2_log;
        b.l3_log = sv->l3_log;
        b.workers = sv->workers;
        b.timeout_ns = (unsigned long long)cfg.timeout_ms * 1000000ull;
        void *p_done = nullptr;
        rc = cuda_fail(cudaHostGetDevicePointer(&p_done, sv->h_done, 0), "map done");
        sp.cmd = sv->d_cmd;
        sp.done = (SlotCompletion *)p_done;
        sp.shutdown = sv->d_shutdown;
        sp.dist = sv->d_dist;
        sp.l2 = sv->d_l2;
        sp.l3 = sv->d_l3;
        sp.l3bits = sv->d_l3bits;
        sp.bits_words = sv->bits_words;
        sp.ctl = sv->d_ctl;
        sp.cta_slot = sv->d_cta_slot;
        sp.slot_first = sv->d_slot_first;
        sp.slots = sv->slots;
        sp.max_n = max_vertices;
        sp.lifetime_ns = (unsigned long long)lifetime_ms * 1000000ull;
        sp.meet_ns = SRV_MEET_NS;
        sp.absent_cta = -1;
        // Test hooks of the bounded slot barrier (tests/test_gpu_server.py).
        if (const char *e = std::getenv("MLMQ_SERVER_MEET_MS"))
            if (std::atoi(e) > 0) sp.meet_ns = (unsigned long long)std::atoi(e) * 1000000ull;
        if (const char *e = std::getenv("MLMQ_SERVER_TEST_ABSENT_CTA")) sp.absent_cta = std::atoi(e);
        if (!rc) {
            cudaLaunchConfig_t lc = {};
            lc.gridDim = dim3((unsigned)sv->grid);
            lc.blockDim = dim3((unsigned)threads);
            lc.dynamicSmemBytes = smem;
            lc.stream = sv->kstream;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeCooperative;
            attr[0].val.cooperative = 1;
            lc.attrs = attr;
            lc.numAttrs = 1;
            void *args[] = {&sp};
            rc = cuda_fail(cudaLaunchKernelExC(&lc, kern, args), "server launch");
        }
        if (!rc) rc = cuda_fail(cudaEventRecord(sv->kdone, sv->kstream), "server event");
        sv->running = !rc;
    }
    if (rc) {
        mlmq_server_destroy(sv);
        return rc;
    }
    *out = sv;
    return MLMQ_OK;
}

}  // namespace

extern "C" int mlmq_server_create(int slots, int max_vertices, const mlmq_config *cfg,
                                  int lifetime_ms, mlmq_server **out) {
    return server_create(slots, nullptr, max_vertices, cfg, lifetime_ms, out);
}

extern "C" int mlmq_server_create_layout(int slots, const int *slot_ctas, int max_vertices,
                                         const mlmq_config *cfg, int lifetime_ms,
                                         mlmq_server **out) {
    if (!slot_ctas) return MLMQ_ERR_ARG;
    return server_create(slots, slot_ctas, max_vertices, cfg, lifetime_ms, out);
}

extern "C" int mlmq_server_layout(const mlmq_server *sv, int *slot_ctas, int max, int *count) {
    if (!sv || !count || (max > 0 && !slot_ctas)) return MLMQ_ERR_ARG;
    const int n = (int)sv->slot_ctas.size();
    for (int s = 0; s < n && s < max; s++) slot_ctas[s] = sv->slot_ctas[s];
    *count = n;
    return MLMQ_OK;
}

extern "C" int mlmq_server_info(const mlmq_server *sv, int *slots, int *grid, int *block) {
    if (!sv) return MLMQ_ERR_ARG;
    if (slots) *slots = sv->slots;
    if (grid) *grid = sv->grid;
    if (block) *block = 32 * (sv->workers + 1);
    return MLMQ_OK;
}

extern "C" int mlmq_server_submit_cfg(mlmq_server *sv, const mlmq_graph *g, int src,
                                      const mlmq_config *knobs, int *h_out, uint64_t *ticket) {
    if (!sv || !g || !h_out || !ticket || src < 0 || src >= g->n || g->slots() > sv->max_n)
        return MLMQ_ERR_ARG;
    if (g->device != sv->device) return MLMQ_ERR_ARG;
    const mlmq_config &k = knobs ? *knobs : sv->cfg;
    if (k.delta < 1 || k.topup < 0 || k.topup > 32 || k.l1_ahead < 0 || k.bucket_max < 1 ||
        k.bucket_max > sv->cfg.bucket_num || (k.bucket_sync != 0 && k.bucket_sync != 1) ||
        (k.light_heavy != 0 && k.light_heavy != 1) || (k.light_heavy && !sv->cfg.vertex_tiles) ||
        g->slots() + (k.light_heavy ? g->n : 0) > sv->max_n)
        return MLMQ_ERR_ARG;
    // Light arcs of this graph for this query's delta.  The running server
    // holds every SM, so nothing can be computed now: they must have been
    // prepared (mlmq_graph_prepare_light) before the server started.
    const int *split = nullptr;
    if (k.light_heavy) {
        const int rc = graph_light_split_cached(g, k.delta, &split);
        if (rc) return rc;
    }
    // Likewise the wide tiles (mlmq_graph_prepare_tiles).
    const int4 *tiles = nullptr;
    int stride = 2;
    if (int rc = graph_tiles_cached(g, sv->cfg.vertex_tiles, &tiles, &stride)) return rc;
    // The smallest free slot with at least the CTAs the query asks for
    // (knobs->work_blocks; 0 or no knobs: any).
    const int want = knobs ? knobs->work_blocks : 0;
    std::lock_guard<std::mutex> lk(sv->mu);
    if (!sv->running) return MLMQ_ERR_STATE;
    int free_slot = -1;
    for (int s = 0; s < sv->slots; s++) {
        auto &c = sv->st[s];
        if (!c.busy && !c.lost && sv->h_done[s].lost) c.lost = true;
        if (!c.busy && !c.lost && sv->slot_ctas[s] >= want &&
            (free_slot < 0 || sv->slot_ctas[s] < sv->slot_ctas[free_slot]))
            free_slot = s;
    }
    if (free_slot < 0) return MLMQ_ERR_BUSY;
    auto &sl = sv->st[free_slot];
    SlotCommand &cmd = sv->h_cmd[free_slot];
    cmd.row = g->d_row;
    cmd.arcs = g->d_arcs;
    cmd.tiles = tiles;
    cmd.n = g->n;
    cmd.nslots = g->slots();
    cmd.src = src;
    cmd.delta = (unsigned)k.delta;
    cmd.topup = k.topup;
    cmd.l1_ahead = k.l1_ahead;
    cmd.bm = k.bucket_max;
    cmd.bucket_sync = k.bucket_sync;
    cmd.split = split;
    cmd.nids = g->slots() + (k.light_heavy ? g->n : 0);
    std::atomic_thread_fence(std::memory_order_release);
    sl.seq++;
    sl.busy = true;
    sl.copying = false;
    sl.ticket = sv->next_ticket++;
    sl.h_out = h_out;
    sl.n = g->n;
    graph_retain(g);  // dropped when the query's result is reported
    sl.g = g;
    cmd.seq = sl.seq;
    // Fields first, then the sequence number: in one stream the second copy
    // starts after the first has landed.  The staging entry is not written
    // again before the slot has taken this command (it is busy until then).
    constexpr size_t head = sizeof(cmd.seq);
    char *dst = reinterpret_cast<char *>(sv->d_cmd + free_slot);
    const char *src_b = reinterpret_cast<const char *>(&cmd);
    int rc = cuda_fail(cudaMemcpyAsync(dst + head, src_b + head, sizeof(SlotCommand) - head,
                                       cudaMemcpyHostToDevice, sv->qstream), "command fields");
    if (!rc) rc = cuda_fail(cudaMemcpyAsync(dst, src_b, head, cudaMemcpyHostToDevice, sv->qstream),
                            "command sequence");
    if (rc) {
        sl.busy = false;
        graph_release(sl.g);
        sl.g = nullptr;
        return rc;
    }
    *ticket = sl.ticket;
    return MLMQ_OK;
}

extern "C" int mlmq_server_submit(mlmq_server *sv, const mlmq_graph *g, int src, int *h_out,
                                  uint64_t *ticket) {
    return mlmq_server_submit_cfg(sv, g, src, nullptr, h_out, ticket);
}

// Moves finished solves to the copy stream and retires finished copies.
extern "C" int mlmq_server_poll(mlmq_server *sv, uint64_t *tickets, int *statuses, int max,
                                int *count) {
    return mlmq_server_poll_timed(sv, tickets, statuses, nullptr, max, count);
}

namespace {

// Advances the slots (see mlmq_server_poll_timed) and reports up to `max`
// finished queries through `emit(index, finished)`.
template <class Emit>
int server_poll(mlmq_server *sv, int max, int *count, Emit emit) {
    std::lock_guard<std::mutex> lk(sv->mu);
    int rc = MLMQ_OK;
    // Whether the server kernel has ended (lifetime, shutdown or an error):
    // queries it never completed are then reported as failed.
    const bool ended = sv->running ? cudaEventQuery(sv->kdone) == cudaSuccess : true;
    for (int s = 0; s < sv->slots; s++) {
        auto &sl = sv->st[s];
        if (!sl.busy) continue;
        if (!sl.copying) {
            if (sv->h_done[s].seq != sl.seq) {
                // No completion: the slot stopped serving (its CTAs could not
                // meet) or the kernel is gone.  The query fails; its host
                // buffer was not written.
                const bool lost = sv->h_done[s].lost != 0;
                if (lost || ended) {
                    sl.lost = sl.lost || lost;
                    sl.busy = false;
                    graph_release(sl.g);
                    sl.g = nullptr;
                    sv->finished.push_back(
                        {sl.ticket, lost ? MLMQ_ERR_TIMEOUT : MLMQ_ERR_STATE, 0ull, 0ull});
                }
                continue;
            }
            std::atomic_thread_fence(std::memory_order_acquire);
            sl.status = sv->h_done[s].status;
            sl.relaxed = sv->h_done[s].relaxed;
            sl.solve_ns = sv->h_done[s].t_end - sv->h_done[s].t_start;
            sl.digest = sv->h_done[s].digest;
            if (sl.status & ST_SLOT_LOST) sl.lost = true;
            rc = cuda_fail(cudaMemcpyAsync(sl.h_out, sv->d_dist + (size_t)s * sv->max_n,
                                           sizeof(int) * (size_t)sl.n, cudaMemcpyDeviceToHost,
                                           sv->cstream), "server D2H");
            if (!rc) rc = cuda_fail(cudaEventRecord(sl.copied, sv->cstream), "copy event");
            if (rc) return rc;
            sl.copying = true;
        } else if (cudaEventQuery(sl.copied) == cudaSuccess) {
            sl.busy = false;
            sl.copying = false;
            graph_release(sl.g);
            sl.g = nullptr;
            sv->finished.push_back({sl.ticket, status_to_error(sl.status), sl.solve_ns, sl.digest});
        }
    }
    int k = 0;
    while (k < max && !sv->finished.empty()) {
        emit(k, sv->finished.front());
        sv->finished.pop_front();
        k++;
    }
    *count = k;
    // The server kernel ending early (lifetime or an error) is reported too.
    if (ended) sv->running = false;
    return MLMQ_OK;
}

}  // namespace

extern "C" int mlmq_server_poll_timed(mlmq_server *sv, uint64_t *tickets, int *statuses,
                                      uint64_t *solve_ns, int max, int *count) {
    if (!sv || !count || (max > 0 && (!tickets || !statuses))) return MLMQ_ERR_ARG;
    return server_poll(sv, max, count, [&](int k, const mlmq_server::Finished &f) {
        tickets[k] = f.ticket;
        statuses[k] = f.status;
        if (solve_ns) solve_ns[k] = f.solve_ns;
    });
}

extern "C" int mlmq_server_poll_results(mlmq_server *sv, mlmq_served_result *out, int max,
                                        int *count) {
    if (!sv || !count || (max > 0 && !out)) return MLMQ_ERR_ARG;
    return server_poll(sv, max, count, [&](int k, const mlmq_server::Finished &f) {
        out[k].ticket = f.ticket;
        out[k].status = f.status;
        out[k].solve_ns = f.solve_ns;
        out[k].digest = f.digest;
    });
}

extern "C" uint64_t mlmq_dist_digest(const int *dist, int64_t n) {
    if (!dist || n <= 0) return 0;
    unsigned long long sum = 0;
    for (int64_t v = 0; v < n; v++) sum += digest_term((unsigned long long)v, dist[v]);
    return sum;
}

extern "C" int mlmq_server_busy_slots(mlmq_server *sv, int *busy) {
    if (!sv || !busy) return MLMQ_ERR_ARG;
    std::lock_guard<std::mutex> lk(sv->mu);
    int b = 0;
    for (auto &sl : sv->st) b += sl.busy || sl.lost;
    *busy = b;
    return sv->running ? MLMQ_OK : MLMQ_ERR_STATE;
}

extern "C" int mlmq_server_stop(mlmq_server *sv) {
    if (!sv) return MLMQ_ERR_ARG;
    int rc = MLMQ_OK;
    if (sv->h_shutdown && sv->d_shutdown && sv->qstream) {
        *(volatile unsigned *)sv->h_shutdown = 1;
        rc = cuda_fail(cudaMemcpyAsync(sv->d_shutdown, sv->h_shutdown, sizeof(unsigned),
                                       cudaMemcpyHostToDevice, sv->qstream), "shutdown flag");
        if (!rc) rc = cuda_fail(cudaStreamSynchronize(sv->qstream), "shutdown flag sync");
    }
    if (sv->kstream) {
        const int krc = cuda_fail(cudaStreamSynchronize(sv->kstream), "server stop");
        if (!rc) rc = krc;
    }
    if (sv->cstream) cudaStreamSynchronize(sv->cstream);
    sv->running = false;
    return rc;
}

extern "C" void mlmq_server_destroy(mlmq_server *sv) {
    if (!sv) return;
    mlmq_server_stop(sv);  // the kernel has ended and result copies are done
    for (auto &sl : sv->st) {
        if (sl.copied) cudaEventDestroy(sl.copied);
        graph_release(sl.g);
        sl.g = nullptr;
    }
    const size_t ns = (size_t)sv->slots;
    cudaStream_t ks = sv->kstream;
    dev_free(sv->d_dist, ks);
    dev_free(sv->d_l2, ks);
    dev_free(sv->d_l3, ks);
    dev_free(sv->d_l3bits, ks);
    dev_free(sv->d_ctl, ks);
    dev_free(sv->d_cta_slot, ks);
    dev_free(sv->d_slot_first, ks);
    dev_free(sv->d_cmd, ks);
    dev_free(sv->d_shutdown, ks);
    pinned_free(sv->h_cmd, sizeof(SlotCommand) * ns);
    pinned_free(sv->h_done, sizeof(SlotCompletion) * ns);
    pinned_free(sv->h_shutdown, 64);
    if (sv->kdone) cudaEventDestroy(sv->kdone);
    if (sv->kstream) cudaStreamDestroy(sv->kstream);
    if (sv->cstream) cudaStreamDestroy(sv->cstream);
    if (sv->qstream) cudaStreamDestroy(sv->qstream);
    delete sv;
}
