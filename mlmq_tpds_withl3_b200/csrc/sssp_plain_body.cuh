// sssp_plain_body.cuh -- body of the persistent single-source kernel, shared by
// the allocating solver (sssp_plain.cu) and the no-allocation entry point
// (noalloc.cu).  `Arcs` selects how arcs are read (see mlmq_queue.cuh).
//
// One cooperative launch per query (reference: work_block_kernel +
// manage_block_kernel on two streams, SS/SSSP/sssp_run.cu:415-674, whose
// manager only ran if the GPU happened to have a free SM).  Every CTA is
// `workers` worker warps plus one manager warp; the cooperative launch
// guarantees all CTAs are resident, so the in-kernel barriers and the
// manager/worker hand-offs cannot wait on a CTA that never started.
//
// Prologue: fill dist with INT_MAX, clear the L3 vertex bits, reset the queue
// counters, barrier, seed
// the source record into bucket 0, barrier.  Then workers loop
// L1 -> L2 window -> L3 -> relax, and manager warps mirror the counters into
// shared memory; CTA 0's manager also detects termination and moves `first`.
#pragma once

#include "mlmq_queue.cuh"

namespace mlmq {

__device__ __forceinline__ void manager_loop(const PlainParams &p, volatile Mirror &mir,
                                             unsigned long long deadline, bool controller) {
    const int lane = threadIdx.x & 31;
    const int rings = p.nb + 1;  // buckets + urgent ring
    const unsigned cap8 = 1u << (p.l2_log - 3);
    unsigned ns = 64;
    for (;;) {
        // Credit is read (acquire) before the reserve counters: a credit is
        // returned only after the pushes it covers, so any credit seen here
        // comes with its reserves and the difference can only overstate the
        // outstanding work.
        const unsigned credit = controller ? ld_acquire(p.ctlw + ctl::CREDIT) : 0u;
        unsigned res = 0, clm = 0, con = 0;
        if (lane < rings) {
            res = ld_relaxed(p.ctlw + ctl::RESERVE + lane);
            clm = ld_relaxed(p.ctlw + ctl::CLAIM + lane);
            con = ld_relaxed(p.ctlw + ctl::CONSUMED + lane);
        }
        const unsigned first = ld_relaxed(p.ctlw + ctl::FIRST);
        const unsigned pres = ld_relaxed(p.ctlw + ctl::PRESSURE);
        const unsigned upres = ld_relaxed(p.ctlw + ctl::U_PRESSURE);
        const unsigned l3r = ld_relaxed(p.ctlw + ctl::L3_RESERVE);
        const unsigned l3c = ld_relaxed(p.ctlw + ctl::L3_CLAIM);
        const unsigned l3k = ld_relaxed(p.ctlw + ctl::L3_CONSUMED);
        const unsigned l3e = ld_relaxed(p.ctlw + ctl::L3_EPOCH);
        unsigned ex = ld_relaxed(p.ctlw + ctl::EXIT);
        if (lane < rings) {
            mir.reserve[lane] = res;
            mir.claim[lane] = clm;
            mir.consumed[lane] = con;
        }
        if (lane == 0) {
            mir.first = first;
            mir.pressure = pres;
            mir.u_pressure = upres;
            mir.l3_reserve = l3r;
            mir.l3_claim = l3c;
            mir.l3_consumed = l3k;
            mir.l3_epoch = l3e;
        }
        if (controller && !ex) {
            unsigned sum = lane < rings ? res : 0u;
            unsigned wait = lane < p.nb ? res - con : 0u;
            unsigned taken = lane < rings ? con : 0u;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                sum += __shfl_xor_sync(FULL, sum, o);
                wait += __shfl_xor_sync(FULL, wait, o);
                taken += __shfl_xor_sync(FULL, taken, o);
            }
            // Records taken from L2/L3 whose work is not finished (credit was
            // read first, so this can only overstate).
            const unsigned in_flight = taken + l3k - credit;
            if (sum + l3r == credit) {
                if (lane == 0) {
                    atomicOr(p.ctlw + ctl::STATUS, ST_DONE);
                    st_release(p.ctlw + ctl::EXIT, 1u);
                }
                ex = 1;
            } else if (sum + l3r - credit == l3r - l3k && l3e != l3r) {
                // Everything outstanding is unread in L3 (no L2 record, no
                // warp holding work): open an L3 epoch.  The window moves up
                // to the smallest distance pushed to L3 since the last one.
                if (lane == 0) {
                    const unsigned m = atomicExch(p.ctlw + ctl::L3_MIN, 0xffffffffu);
                    if (m != 0xffffffffu) atomicMax(p.ctlw + ctl::FIRST, m / p.delta);
                    st_release(p.ctlw + ctl::L3_EPOCH, l3r);
                }
            } else {
                // Urgent records (below the window) still to be read.
                const unsigned urgent = __shfl_sync(FULL, res - con, p.nb);
                if (wait != 0 && urgent == 0 && (!p.bucket_sync || in_flight == 0)) {
                    // Move `first` towards the first non-empty bucket of the
                    // window, one bucket per step (as the reference's readers
                    // do): a bucket whose records were all taken may still be
                    // producing records in warps' L1 rings, and a window that
                    // runs ahead of them turns their results into urgent
                    // corrections of work already done.
                    const int b = (int)((first + (unsigned)lane) % (unsigned)p.nb);
                    const unsigned rb = __shfl_sync(FULL, res, b);
                    const unsigned cb = __shfl_sync(FULL, con, b);
                    const unsigned ne = __ballot_sync(FULL, lane < p.nb && rb != cb);
                    const int i0 = ne ? __ffs(ne) - 1 : 0;
                    // With bucket sync nothing is in flight, so the window
                    // may jump straight to the first non-empty bucket.
                    const unsigned step = p.bucket_sync ? (unsigned)i0 : 1u;
                    if (i0 > 0 && lane == 0) atomicMax(p.ctlw + ctl::FIRST, first + step);
                }
                // Release bucket pressure once the ring has drained.
                if (lane < p.nb && ((pres >> lane) & 1u) && res - con < cap8)
                    atomicAnd(p.ctlw + ctl::PRESSURE, ~(1u << lane));
                if (lane == p.nb && res - con < cap8 && ld_relaxed(p.ctlw + ctl::U_PRESSURE))
                    st_relaxed(p.ctlw + ctl::U_PRESSURE, 0u);
            }
        }
        if (!ex && globaltimer() > deadline) {
            if (lane == 0) raise_status(p, ST_TIMEOUT);
            ex = 1;
        }
        ex = __shfl_sync(FULL, ex, 0);
        if (ex) {
            if (lane == 0) mir.exit = 1;
            return;
        }
        __nanosleep(ns);
        if (ns < 256) ns <<= 1;
    }
}

template <class Arcs, int K, bool kSplit>
__device__ __forceinline__ void worker_loop(const PlainParams &p, volatile Mirror &mir, uint2 *ring,
                                            uint2 *inb, int2 *stage, WarpQ &q) {
    const int lane = threadIdx.x & 31;
    for (;;) {
        if (mir.exit) break;
        if (p.l1_ahead) {
            const unsigned long long lim =
                ((unsigned long long)mir.first + (unsigned)p.l1_ahead) * p.delta;
            q.l1_lim = lim < 0xffffffffull ? (unsigned)lim : 0xffffffffu;
        }
        bool valid = false;
        unsigned v = 0, d = 0;
        if (q.l1_size > 0) {
            const int k = q.l1_size < 32 ? q.l1_size : 32;
            l1_read(q, ring, valid, v, d);
            if (k < p.topup && l2_has_work(p, q, mir)) {
                // Few records in L1: fill the rest of the warp from the L2
                // window, so an iteration relaxes a full warp of records.
                const int got = l2_read(p, q, mir, inb, 32 - k, 32 - k);
                if (got) {
                    q.onfly += (unsigned)got;
                    __syncwarp();
                    if (lane >= k && lane < k + got) {
                        const uint2 it = inb[lane - k];
                        valid = true;
                        v = it.x;
                        d = it.y;
                    }
                    __syncwarp();
                }
            }
        } else {
            if (q.ob_n) outbox_flush(p, q, ring, true);
            int got = l2_has_work(p, q, mir) ? l2_read(p, q, mir, inb, 32, p.min_read) : 0;
            if (got == 0 && q.onfly) {
                // L1 and the outbox are empty and L2 has nothing for this
                // warp: everything derived from the records read so far is
                // reserved in L2/L3, so their credit may go back.  A warp
                // that finds more records keeps its credit and returns it
                // with theirs, which takes the fence off the busy path
                // (R-MAT-22 +3 %); a warp always reads L2 before it idles,
                // so credit is never held by an idle warp.
                __threadfence();
                __syncwarp();
                if (lane == 0) atomicAdd(p.ctlw + ctl::CREDIT, q.onfly);
                q.onfly = 0;
            }
            if (got == 0) {
                // Nothing in L2: re-bucket L3 records if an epoch is open.
                // Their credit is returned once L1 is empty, after the
                // pushes that re-bucketed them.
                const int moved = l3_rebucket<kSplit>(p, q, mir);
                if (moved) {
                    q.onfly += (unsigned)moved;
                    q.idle_ns = 32;
                    continue;
                }

                if constexpr (kStatsSmem) wstat_add(WS_IDLE, 1u);
                else q.idle++;
                __nanosleep(q.idle_ns);
                if (q.idle_ns < 256) q.idle_ns <<= 1;
                continue;
            }
            q.idle_ns = 32;
            q.onfly += (unsigned)got;
            __syncwarp();
            valid = lane < got;
            if (valid) {
                const uint2 it = inb[lane];
                v = it.x;
                d = it.y;
            }
            __syncwarp();
        }
        if constexpr (kStatsSmem) wstat_add(WS_BATCHES, 1u);
        else q.batches++;
        relax_batch<Arcs, K, kSplit>(p, q, ring, stage, valid, v, d);
    }
}

// `grank`/`gsize`: this CTA's rank in, and the size of, the group of CTAs
// that serves the query (the whole grid for a single-source launch).  K is
// the number of 32-arc relaxation rounds a warp keeps in flight; kSplit as
// for relax_batch (true whenever the graph has pieces or light_heavy is on).
template <class Arcs, int K, bool kSplit = true>
__device__ __forceinline__ void plain_body(const PlainParams &p, unsigned grank, unsigned gsize) {
    extern __shared__ uint2 smem[];
    volatile Mirror &mir = cta_mirror;
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const unsigned long long deadline = globaltimer() + p.timeout_ns;

    // ---- prologue: reset ------------------------------------------------------
    const size_t gtid = (size_t)grank * blockDim.x + threadIdx.x;
    const size_t gstride = (size_t)gsize * blockDim.x;
    for (size_t i = gtid; i < (size_t)p.n; i += gstride) p.dist[i] = INT_MAX;
    for (size_t i = gtid; i < ((size_t)p.nids + 31) / 32; i += gstride) p.l3bits[i] = 0u;
    if (grank == 0) {
        for (int i = threadIdx.x; i < ctl::WORDS; i += blockDim.x)
            if (i != ctl::BAR_COUNT && i != ctl::BAR_GEN) p.ctlw[i] = 0u;
    }
    if (!grid_barrier(p.ctlw, gsize, deadline)) return;
    if (grank == 0 && threadIdx.x == 0) {
        p.dist[p.src] = 0;
        *l2_slot(p, 0, 0u) = rec_pack((unsigned)p.src, 0u, 0u);
        p.ctlw[ctl::RESERVE + 0] = 1u;
        p.ctlw[ctl::L3_MIN] = 0xffffffffu;
        p.ctlw[ctl::STATS + 2 * ctl::ST_PUSHED] = 1u;
    }
    if (!grid_barrier(p.ctlw, gsize, deadline)) return;

    // ---- initial mirror ----------------------------------------------------------
    if (threadIdx.x < NB_MAX) {
        mir.reserve[threadIdx.x] = ld_relaxed(p.ctlw + ctl::RESERVE + threadIdx.x);
        mir.claim[threadIdx.x] = 0u;
        mir.consumed[threadIdx.x] = 0u;
    }
    if (threadIdx.x == 0) {
        mir.first = 0u;
        mir.exit = 0u;
        mir.pressure = 0u;
        mir.u_pressure = 0u;
        mir.l3_reserve = mir.l3_claim = mir.l3_consumed = mir.l3_epoch = 0u;
    }
    __syncthreads();

    if (warp == p.workers) {
        manager_loop(p, mir, deadline, grank == 0);
        return;
    }

    uint2 *ring = smem + (size_t)warp * WARP_SMEM_SLOTS;
    uint2 *inb = ring + L1_CAP;
    int2 *stage = reinterpret_cast<int2 *>(inb + 32);
    WarpQ q;
    q.l1_head = q.l1_tail = q.l1_size = 0;
    q.ob_n = 0;
    q.l1_lim = 0xffffffffu;
    q.c_lo = q.c_hi = 0u;
    q.l3_lo = q.l3_hi = 0u;
    q.onfly = 0u;
    q.idle_ns = 32u;
    q.range_hit = 0u;
    q.pushed = q.l3_pushed = q.relaxed = q.improved = 0ull;
    q.batches = q.idle = 0u;
    q.deadline = deadline;
    if constexpr (kStatsSmem) {
        if (lane < 8) wstat()[lane] = lane == WS_DEADLINE ? deadline : 0ull;
        __syncwarp();
    }

    worker_loop<Arcs, K, kSplit>(p, mir, ring, inb, stage, q);

    // ---- epilogue: statistics --------------------------------------------------
    unsigned long long pushed, l3_pushed, relaxed, improved, batches, idle;
    bool range;
    if constexpr (kStatsSmem) {
        __syncwarp();
        const unsigned long long *ws = wstat();
        pushed = ws[WS_PUSHED];
        l3_pushed = ws[WS_L3_PUSHED];
        relaxed = ws[WS_RELAXED];
        improved = ws[WS_IMPROVED];
        batches = ws[WS_BATCHES];
        idle = ws[WS_IDLE];
        range = ws[WS_RANGE] != 0ull;
    } else {
        pushed = q.pushed;
        l3_pushed = q.l3_pushed;
        relaxed = q.relaxed;
        improved = q.improved;
        batches = q.batches;
        idle = q.idle;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            relaxed += __shfl_xor_sync(FULL, relaxed, o);
            improved += __shfl_xor_sync(FULL, improved, o);
        }
        range = __ballot_sync(FULL, q.range_hit != 0u) != 0u;
    }
    if (lane == 0) {
        unsigned long long *st = reinterpret_cast<unsigned long long *>(p.ctlw + ctl::STATS);
        atomicAdd(st + ctl::ST_PUSHED, pushed);
        atomicAdd(st + ctl::ST_L3_PUSHED, l3_pushed);
        atomicAdd(st + ctl::ST_RELAXED, relaxed);
        atomicAdd(st + ctl::ST_IMPROVED, improved);
        atomicAdd(st + ctl::ST_BATCHES, batches);
        atomicAdd(st + ctl::ST_IDLE, idle);
        if (range) atomicOr(p.ctlw + ctl::STATUS, ST_RANGE);
        atomicMax(st + ctl::ST_FIRST_MAX, (unsigned long long)ld_relaxed(p.ctlw + ctl::FIRST));
    }
}

}  // namespace mlmq
