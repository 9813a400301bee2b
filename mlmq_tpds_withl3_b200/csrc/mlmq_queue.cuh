// mlmq_queue.cuh -- the three-level MLMQ work queue and the CSR relaxation
// step, as warp-cooperative device functions used by the persistent kernel.
//
// Reference behaviour restated here (hideoze/mlmq_tpds_withl3):
//  * L1 SLF queue, core/src/l1_queue.cu:218-360: a 64-slot ring per warp in
//    shared memory; an incoming record goes to the FRONT when its distance is
//    below the front record's (or, with the ring empty, below the first
//    incoming record's), otherwise to the BACK; when the ring holds more than
//    32 records every record spills to L2; reads take up to 32 from the front.
//  * L2 delta buckets, core/cu_delta_queue/cu_delta_queue.cuh:78-642: BNUM
//    circular buckets of width delta starting at bucket `first`; writers
//    reserve slots with one warp-aggregated atomicAdd per destination bucket
//    (__match_any_sync); readers claim l2_batch_size slots per bucket from up
//    to BUCKET_MAX buckets starting at `first`, keep a claim they could not
//    finish, and stop once MIN_READ_GRA records are held; `first` moves on
//    once its bucket is empty and other buckets still hold records.
//  * Relaxation, SS/SSSP/sssp_run.cu:143-413: stale records (distance above
//    the vertex's current distance) are dropped; vertices of out-degree >=
//    LARGEV are relaxed by the whole warp, smaller ones through a warp prefix
//    sum over degrees that gives every lane one arc; atomicMin on int32
//    distances; winners are ballot-compacted into the queue.
//  * Termination, sssp_run.cu:565-572 and :644-661: a warp returns the read
//    credit of its L2 records only when its L1 is empty, and the solve ends
//    when (records reserved) - (credit returned) reaches zero.
//
// Where the B200 design differs (each a deliberate change, not a port):
//  * Publication without manager warps.  A ring slot is one 64-bit word
//    holding the record plus a 2-bit lap tag; the writer installs it with one
//    atomicCAS from the empty word, so a reader knows a slot is readable from
//    the slot alone and clears it after reading.  The reference needed
//    per-512-record write counters and 16 manager warps to publish read_pos.
//  * Per-CTA mirror.  One warp per CTA copies the queue counters into shared
//    memory; worker warps poll that copy instead of global memory, so idle
//    warps add no global traffic.
//  * Urgent bucket.  A record whose distance is below the window start (it
//    was produced while `first` moved on) goes to one extra ring that readers
//    visit first, instead of being clamped into bucket `first`, whose ring
//    may already stand for a far bucket.
//  * L3.  Records beyond the bucket window (the reference clamps them into
//    the last bucket) and records for a bucket whose ring is filling go to
//    one HBM ring shared by every CTA.  Warps read it when every L2 bucket is
//    empty and move `first` up to the batch they took.  L3 keeps at most one
//    record per vertex: a per-vertex bit marks "has an L3 record", a push
//    finding the bit set is dropped, and an L3 record is relaxed with the
//    vertex's distance at read time (never filtered as stale), so the
//    dropped improvement is applied.  L3 therefore never holds more than n
//    records plus the pushes in flight, which bounds every queue level.
//  * Every wait is bounded by a deadline and ends with a status bit, never a
//    trap or an endless spin.
#pragma once

#include "device_common.cuh"

namespace mlmq {

struct PlainParams {
    int n;
    int nslots;  // n + split-vertex pieces (ids n .. nslots-1 are pieces)
    int nids;    // nslots, + n with the light/heavy split (ids nslots + v: v's heavy record)
    const int *__restrict__ row;
    const int2 *__restrict__ arcs;  // interleaved {dst, weight} (ArcsInterleaved)
    const int4 *__restrict__ tiles; // tile_stride per vertex, or null: read row offsets instead
    int tile_stride;                // int4 per tile: 2 (4 inline arcs) or 4 (8 inline arcs)
    const int *__restrict__ col;    // caller's CSR arrays, read in place (ArcsSplit)
    const int *__restrict__ w;
    int *dist;
    int src;
    unsigned long long *l2;  // (nb + 1) rings of 2^l2_log slots; ring nb is the urgent ring
    unsigned long long *l3;  // 2^l3_log slots
    unsigned *l3bits;        // one bit per vertex: the vertex has a record in L3
    unsigned *ctlw;
    int nb, bm, batch, min_read, large, l1_spill, l1_vector;
    int l1_keep;   // records kept at the L1 front when it spills (0: spill all)
    int l1_ahead;  // buckets past `first` a winner may be to stay in L1 (0: no limit)
    int topup;     // fewer than this many L1 records: fill the warp from L2 too
    int bucket_sync;  // 1: `first` advances only when no taken record is still in flight
    const int *__restrict__ split;  // light arcs (w < delta) per vertex, or null: no split
    int precheck;  // read dist[dst] before the atomicMin
    unsigned delta;
    int l2_log, l3_log;
    int workers;  // worker warps per CTA (one more warp per CTA is the manager)
    unsigned long long timeout_ns;
};

// Shared-memory copy of the global queue counters, refreshed by the manager
// warp of each CTA.
struct Mirror {
    unsigned first, exit, pressure, u_pressure;
    unsigned l3_reserve, l3_claim, l3_consumed, l3_epoch;
    unsigned reserve[NB_MAX], claim[NB_MAX], consumed[NB_MAX];
};
// The CTA's mirror: one per CTA in static shared memory, so that the queue
// functions can read it without a pointer passed down every call.
static __shared__ Mirror cta_mirror;

// Per-warp queue state held in registers.  l1_* and the L3 claim are
// warp-uniform; c_lo/c_hi are lane-distributed (lane b: claim on ring b).
struct WarpQ {
    int l1_head, l1_tail, l1_size;
    int ob_n;  // records in the outbox (ring + OUTBOX_OFF)
    unsigned c_lo, c_hi;
    unsigned l3_lo, l3_hi;
    unsigned onfly;
    unsigned l1_lim;  // winners at or above this distance skip L1 (bucket window)
    unsigned idle_ns;
    unsigned range_hit;
    unsigned long long pushed, l3_pushed, relaxed, improved;
    unsigned batches, idle;  // warp iterations with records / without (warp-uniform)
    unsigned long long deadline;
};

// Where the per-warp counters (pushed, relaxed, ... and the deadline) live.
// A translation unit that defines MLMQ_WARP_STATS_SMEM to 1 before including
// this header keeps them in the warp's shared-memory block (WSTAT_OFF), warp
// totals added by lane 0, and the WarpQ fields above go unused: the batched
// and served kernels hold per-query parameters too, and the registers this
// frees let four CTAs of nine warps share an SM instead of three
// (measured: 64 batched grid queries 338 -> 392 queries/s).  Single solves
// keep them in registers, where the counters cost no instructions on the
// chain of dependent hops.
#ifndef MLMQ_WARP_STATS_SMEM
#define MLMQ_WARP_STATS_SMEM 0
#endif
constexpr bool kStatsSmem = MLMQ_WARP_STATS_SMEM != 0;

__device__ __forceinline__ unsigned long long *wstat() {
    extern __shared__ uint2 smem[];
    return reinterpret_cast<unsigned long long *>(smem + (size_t)(threadIdx.x >> 5) * WARP_SMEM_SLOTS +
                                                  WSTAT_OFF);
}
// Adds a warp-uniform amount to shared-memory counter i (lane 0 adds).
__device__ __forceinline__ void wstat_add(int i, unsigned x) {
    if ((threadIdx.x & 31) == 0 && x) atomicAdd(wstat() + i, (unsigned long long)x);
}
__device__ __forceinline__ unsigned long long warp_deadline(const WarpQ &q) {
    if constexpr (kStatsSmem) return wstat()[WS_DEADLINE];
    else return q.deadline;
}

__device__ __forceinline__ unsigned long long *l2_slot(const PlainParams &p, int ring, unsigned s) {
    return p.l2 + ((size_t)ring << p.l2_log) + (s & ((1u << p.l2_log) - 1u));
}
__device__ __forceinline__ unsigned long long *l3_slot(const PlainParams &p, unsigned s) {
    return p.l3 + (s & ((1u << p.l3_log) - 1u));
}

__device__ __forceinline__ void raise_status(const PlainParams &p, unsigned bits) {
    atomicOr(p.ctlw + ctl::STATUS, bits);
    st_relaxed(p.ctlw + ctl::EXIT, 1u);
}

// Installs a record in a slot still holding the previous lap's record: waits,
// bounded by the deadline, for its reader to clear it.
static __device__ __noinline__ void install_slow(const PlainParams &p, unsigned long long *slot,
                                          unsigned long long rec, unsigned long long deadline) {
    unsigned ns = 64;
    for (;;) {
        __nanosleep(ns);
        if (atomicCAS(slot, SENT, rec) == SENT) return;
        if (ns < 2048) ns <<= 1;
        if (globaltimer() > deadline || ld_relaxed(p.ctlw + ctl::EXIT)) {
            raise_status(p, ST_QUEUE_FULL);
            return;
        }
    }
}

// Warp-cooperative push of up to 32 records (one per lane with `valid`).
// Ring choice: urgent ring for distances below the window, bucket
// floor(d/delta) mod nb inside the window, L3 beyond it or under pressure.
__device__ __forceinline__ void push32(const PlainParams &p, WarpQ &q, bool valid, unsigned v,
                                       unsigned d) {
    if (!__ballot_sync(FULL, valid)) return;
    const int lane = threadIdx.x & 31;
    // The window start and the pressure bits from the CTA's mirror instead
    // of three global loads (one L2 round trip less per push; C3 +5 %).  The
    // global words were read relaxed, i.e. possibly stale, already; a stale
    // value only sends a record to a ring read later or to L3, and every
    // record is relaxed when it comes out.
    volatile Mirror &m = cta_mirror;
    const unsigned f = m.first;
    const unsigned pres = m.pressure;
    const unsigned upres = m.u_pressure;
    int tgt = -1;
    if (valid) {
        const unsigned L = d / p.delta;
        if (L < f) {
            tgt = upres ? NB_MAX : p.nb;  // urgent ring, or L3 while it is filling
        } else if (L - f >= (unsigned)p.nb) {
            tgt = NB_MAX;  // L3
        } else {
            const int b = (int)(L % (unsigned)p.nb);
            tgt = ((pres >> b) & 1u) ? NB_MAX : b;
        }
    }
    if (tgt == NB_MAX) {
        // One L3 record per vertex.  The fence orders the atomicMin that made
        // this record before the bit test: a reader that clears the bit after
        // this atomicOr and then reads dist[v] sees the improvement, so a
        // push dropped here loses nothing.
        __threadfence();
        const unsigned bit = 1u << (v & 31u);
        if (atomicOr(p.l3bits + (v >> 5), bit) & bit) {
            valid = false;
            tgt = -1;
        }
    }
    const unsigned act = __ballot_sync(FULL, valid);
    if (!act) return;
    const unsigned grp = __match_any_sync(FULL, tgt);
    const int leader = __ffs(grp) - 1;
    const unsigned rank = __popc(grp & lanemask_lt());
    const unsigned cnt = __popc(grp);
    unsigned base = 0;
    if (valid && lane == leader) {
        if (tgt < NB_MAX) {
            const unsigned cons = ld_relaxed(p.ctlw + ctl::CONSUMED + tgt);
            base = atomicAdd(p.ctlw + ctl::RESERVE + tgt, cnt);
            // More than half the ring outstanding: later pushes for this ring
            // go to L3 until it drains.  The urgent ring needs this as much
            // as a bucket: every record produced below the window goes
            // there, and a full ring would leave pushers waiting for slots
            // that only other (pushing) warps can free.
            if (base + cnt - cons > (1u << (p.l2_log - 1))) {
                if (tgt < p.nb) atomicOr(p.ctlw + ctl::PRESSURE, 1u << tgt);
                else st_relaxed(p.ctlw + ctl::U_PRESSURE, 1u);
            }
        } else {
            base = atomicAdd(p.ctlw + ctl::L3_RESERVE, cnt);
        }
    }
    base = __shfl_sync(FULL, base, leader);
    if (valid) {
        const unsigned s = base + rank;
        unsigned long long *slot;
        unsigned lap;
        if (tgt < NB_MAX) {
            slot = l2_slot(p, tgt, s);
            lap = s >> p.l2_log;
        } else {
            slot = l3_slot(p, s);
            lap = s >> p.l3_log;
        }
        const unsigned long long rec = rec_pack(v, d, lap);
        if (atomicCAS(slot, SENT, rec) != SENT) install_slow(p, slot, rec, warp_deadline(q));
    }
    const unsigned l3m = __ballot_sync(FULL, valid && tgt == NB_MAX);
    if (l3m) {
        // Where the window goes when the next L3 epoch opens.
        const unsigned dm = __reduce_min_sync(FULL, (valid && tgt == NB_MAX) ? d : 0xffffffffu);
        if (lane == __ffs(l3m) - 1) atomicMin(p.ctlw + ctl::L3_MIN, dm);
    }
    if constexpr (kStatsSmem) {
        wstat_add(WS_PUSHED, __popc(act));
        wstat_add(WS_L3_PUSHED, __popc(l3m));
    } else {
        q.pushed += __popc(act);
        q.l3_pushed += __popc(l3m);
    }
}

// ---- L1: warp-private ring in shared memory ---------------------------------
// SLF insert (l1_queue.cu:284-330) or, for the vector L1, append at the back;
// then spill everything to L2 when more than l1_spill records are held
// (l1_queue.cu:332-350).  At most 32 records per call, so the 64-slot ring
// never overflows.
// Pushes the outbox's records 32 at a time (all of them when `all`, else
// while 32 or more are held).  A warp empties it before it returns its read
// credit, so the solve cannot end with records held here.
__device__ __forceinline__ void outbox_flush(const PlainParams &p, WarpQ &q, uint2 *ring, bool all) {
    const int lane = threadIdx.x & 31;
    uint2 *ob = ring + OUTBOX_OFF;
    while (q.ob_n >= 32 || (all && q.ob_n > 0)) {
        const int k = q.ob_n < 32 ? q.ob_n : 32;
        const int rest = q.ob_n - k;
        const bool ok = lane < k;
        uint2 it = make_uint2(0u, 0u), mv = make_uint2(0u, 0u);
        if (ok) it = ob[lane];
        if (lane < rest) mv = ob[k + lane];
        __syncwarp();
        if (lane < rest) ob[lane] = mv;
        __syncwarp();
        q.ob_n = rest;
        push32(p, q, ok, it.x, it.y);
    }
}

__device__ __forceinline__ void l1_write(const PlainParams &p, WarpQ &q, uint2 *ring, bool valid,
                                         unsigned v, unsigned d) {
    // A winner beyond the bucket window goes to L2/L3, not to this warp's L1:
    // following it here would let the warp's chain of relaxations run ahead
    // of the window on distances that are not final yet, and the real
    // frontier would redo that work later.  Such winners gather in the
    // outbox and are pushed 32 at a time.
    if (q.l1_lim != 0xffffffffu) {
        const bool far = valid && d >= q.l1_lim;
        const unsigned fm = __ballot_sync(FULL, far);
        if (fm) {
            if (far) ring[OUTBOX_OFF + q.ob_n + (int)__popc(fm & lanemask_lt())] = make_uint2(v, d);
            __syncwarp();
            q.ob_n += (int)__popc(fm);
            if (q.ob_n >= 32) outbox_flush(p, q, ring, false);
            valid = valid && !far;
        }
    }
    const unsigned vm = __ballot_sync(FULL, valid);
    if (!vm) return;
    const unsigned front_d =
        q.l1_size > 0 ? ring[q.l1_head].y : __shfl_sync(FULL, d, __ffs(vm) - 1);
    const bool left = valid && !p.l1_vector && d < front_d;
    const unsigned lm = __ballot_sync(FULL, left);
    const unsigned rm = vm & ~lm;
    if (left)
        ring[(q.l1_head - (int)__popc(lm & lanemask_le())) & (L1_CAP - 1)] = make_uint2(v, d);
    else if (valid)
        ring[(q.l1_tail + (int)__popc(rm & lanemask_lt())) & (L1_CAP - 1)] = make_uint2(v, d);
    __syncwarp();
    q.l1_head = (q.l1_head - (int)__popc(lm)) & (L1_CAP - 1);
    q.l1_tail = (q.l1_tail + (int)__popc(rm)) & (L1_CAP - 1);
    q.l1_size += (int)__popc(vm);
    if (q.l1_size > p.l1_spill) {
        // Spill from the back; the l1_keep front (smallest-first) records stay
        // so the warp's own chain of relaxations continues in shared memory.
        const int lane = threadIdx.x & 31;
        const int first = p.l1_keep;
        for (int c = first; c < q.l1_size; c += 32) {
            const int i = c + lane;
            const bool ok = i < q.l1_size;
            uint2 it = make_uint2(0u, 0u);
            if (ok) it = ring[(q.l1_head + i) & (L1_CAP - 1)];
            push32(p, q, ok, it.x, it.y);
        }
        __syncwarp();
        q.l1_tail = (q.l1_head + first) & (L1_CAP - 1);
        q.l1_size = first;
    }
}

// Up to 32 records from the front of L1 (l1_queue.cu:253-273).
__device__ __forceinline__ void l1_read(WarpQ &q, const uint2 *ring, bool &valid, unsigned &v,
                                        unsigned &d) {
    const int lane = threadIdx.x & 31;
    const int k = q.l1_size < 32 ? q.l1_size : 32;
    valid = lane < k;
    if (valid) {
        const uint2 it = ring[(q.l1_head + lane) & (L1_CAP - 1)];
        v = it.x;
        d = it.y;
    }
    __syncwarp();
    q.l1_head = (q.l1_head + k) & (L1_CAP - 1);
    q.l1_size -= k;
}

// Takes the readable prefix of this warp's claim on L2 ring `ring` into
// inb[got...]; returns the number taken.
__device__ __forceinline__ int take_claim(const PlainParams &p, volatile Mirror &mir, int ring,
                                          unsigned &lo, unsigned hi, uint2 *inb, int got, int room) {
    const int lane = threadIdx.x & 31;
    const unsigned res = mir.reserve[ring];
    int ready = (int)(res - lo);
    if (ready <= 0) return 0;
    if (ready > (int)(hi - lo)) ready = (int)(hi - lo);
    if (ready > room - got) ready = room - got;
    unsigned long long r = SENT;
    bool ok = false;
    const unsigned s = lo + lane;
    if (lane < ready) {
        r = ld_relaxed64(l2_slot(p, ring, s));
        ok = (r != SENT) && rec_lap(r) == ((s >> p.l2_log) & 3u);
    }
    const unsigned okm = __ballot_sync(FULL, ok);
    int take = (okm == FULL) ? 32 : (__ffs(~okm) - 1);
    if (take > ready) take = ready;
    if (lane < take) {
        inb[got + lane] = make_uint2(rec_v(r), rec_d(r));
        st_relaxed64(l2_slot(p, ring, s), SENT);
    }
    if (take > 0 && lane == 0) atomicAdd(p.ctlw + ctl::CONSUMED + ring, (unsigned)take);
    lo += (unsigned)take;
    return take;
}

// One ring of the read window: continue a pending claim or make a new one
// (only when the mirror shows unclaimed reserved slots), then take records.
__device__ __forceinline__ int read_ring(const PlainParams &p, WarpQ &q, volatile Mirror &mir,
                                         int ring, uint2 *inb, int got, int room) {
    const int lane = threadIdx.x & 31;
    unsigned lo = __shfl_sync(FULL, q.c_lo, ring);
    unsigned hi = __shfl_sync(FULL, q.c_hi, ring);
    if (lo == hi) {
        if ((int)(mir.reserve[ring] - mir.claim[ring]) <= 0) return 0;
        if (got + p.batch > room) return 0;
        unsigned nlo = 0;
        if (lane == 0) {
            nlo = atomicAdd(p.ctlw + ctl::CLAIM + ring, (unsigned)p.batch);
            atomicMax((unsigned *)&mir.claim[ring], nlo + (unsigned)p.batch);
        }
        lo = __shfl_sync(FULL, nlo, 0);
        hi = lo + (unsigned)p.batch;
    }
    const int t = take_claim(p, mir, ring, lo, hi, inb, got, room);
    if (lane == ring) {
        q.c_lo = lo;
        q.c_hi = hi;
    }
    return t;
}

// Whether an L2 read could find anything: lane r looks at ring r (the urgent
// ring or a bucket of the read window) in the CTA mirror -- unclaimed
// reserved slots, or reserved slots inside this warp's own pending claim.
// Costs one shared-memory read per lane and a vote, so an idle warp can
// poll it instead of running the full read.
__device__ __forceinline__ bool l2_has_work(const PlainParams &p, const WarpQ &q,
                                            volatile Mirror &mir) {
    const int lane = threadIdx.x & 31;
    bool has = false;
    if (lane <= p.nb) {
        const unsigned rel = ((unsigned)lane + (unsigned)p.nb - mir.first % (unsigned)p.nb) %
                             (unsigned)p.nb;
        if (lane == p.nb || rel < (unsigned)p.bm) {
            const unsigned res = mir.reserve[lane];
            has = (int)(res - mir.claim[lane]) > 0 || (q.c_lo != q.c_hi && res != q.c_lo);
        }
    }
    return __any_sync(FULL, has);
}

// L2 read (cu_delta_queue.cuh:272-428 with ml_queue.cu:238-307): urgent ring
// first, then buckets first .. first+bucket_max-1, until `want` records (at
// most `room`) are in inb.
__device__ __forceinline__ int l2_read(const PlainParams &p, WarpQ &q, volatile Mirror &mir,
                                       uint2 *inb, int room, int want) {
    int got = read_ring(p, q, mir, p.nb, inb, 0, room);
    const unsigned f = mir.first;
    for (int i = 0; i < p.bm && got < want; i++) {
        const int b = (int)((f + (unsigned)i) % (unsigned)p.nb);
        got += read_ring(p, q, mir, b, inb, got, room);
    }
    return got;
}

// L3 re-bucketing.  L3 holds records that did not fit the L2 window (beyond
// it, or for a ring under pressure).  Relaxing them as they come out would
// run a second, speculative wavefront far ahead of the real one; instead a
// record goes back through push32 -- into the urgent ring below the window,
// its bucket inside it, or L3 again beyond it -- so it is relaxed in bucket
// order.  Reads happen in epochs: the controller opens one (sets L3_EPOCH to
// the current L3 reserve count and moves `first` to the smallest distance
// pushed to L3 since the last epoch) when everything outstanding is in L3,
// and a warp with nothing else to do takes records from slots below the
// epoch mark only, so each record is re-bucketed at most once per epoch.
// Each taken record's vertex bit is cleared and then the vertex's distance is
// read again: that value covers every L3 push dropped while the record
// waited, and it is the distance the record goes back with.  Returns the
// number of records taken (their read credit).
template <bool kSplit>
__device__ __forceinline__ int l3_rebucket(const PlainParams &p, WarpQ &q, volatile Mirror &mir) {
    const int lane = threadIdx.x & 31;
    unsigned pending = 0;
    if (lane <= p.nb) pending = mir.reserve[lane] - mir.consumed[lane];
    if (__ballot_sync(FULL, pending != 0)) return 0;
    const unsigned epoch = mir.l3_epoch;
    if (q.l3_lo == q.l3_hi) {
        if ((int)(epoch - mir.l3_claim) <= 0) return 0;
        unsigned nlo = 0;
        if (lane == 0) {
            nlo = atomicAdd(p.ctlw + ctl::L3_CLAIM, 32u);
            atomicMax((unsigned *)&mir.l3_claim, nlo + 32u);
        }
        q.l3_lo = __shfl_sync(FULL, nlo, 0);
        q.l3_hi = q.l3_lo + 32u;
    }
    int ready = (int)(min(epoch, mir.l3_reserve) - q.l3_lo);
    if (ready <= 0) return 0;
    if (ready > (int)(q.l3_hi - q.l3_lo)) ready = (int)(q.l3_hi - q.l3_lo);
    const unsigned s = q.l3_lo + lane;
    unsigned long long r = SENT;
    bool ok = false;
    if (lane < ready) {
        r = ld_relaxed64(l3_slot(p, s));
        ok = (r != SENT) && rec_lap(r) == ((s >> p.l3_log) & 3u);
    }
    const unsigned okm = __ballot_sync(FULL, ok);
    int take = (okm == FULL) ? 32 : (__ffs(~okm) - 1);
    if (take > ready) take = ready;
    unsigned v = 0, cur = 0;
    if (lane < take) {
        v = rec_v(r);
        st_relaxed64(l3_slot(p, s), SENT);
        atomicAnd(p.l3bits + (v >> 5), ~(1u << (v & 31u)));
        __threadfence();
        // A piece has no distance of its own: its owner's stands for it; a
        // heavy record stands for its vertex's distance + delta.
        unsigned dv = v, add = 0u;
        if (kSplit && v >= (unsigned)p.nslots) {
            dv = v - (unsigned)p.nslots;
            add = p.delta;
        } else if (kSplit && v >= (unsigned)p.n) {
            dv = (unsigned)__ldg(p.tiles + (size_t)p.tile_stride * v).w;
        }
        const unsigned long long now = (unsigned long long)(unsigned)__ldcg(p.dist + dv) + add;
        cur = (unsigned)min(now, (unsigned long long)rec_d(r));
    }
    if (take > 0 && lane == 0) atomicAdd(p.ctlw + ctl::L3_CONSUMED, (unsigned)take);
    q.l3_lo += (unsigned)take;
    push32(p, q, lane < take, v, cur);
    return take;
}

// ---- relaxation --------------------------------------------------------------
// Arc loaders.  The allocating solver builds one interleaved {dst, weight}
// array so an arc is one 8-byte load; the no-allocation entry point cannot
// build it and reads the caller's ColIdx and edge_data arrays in place.
struct ArcsInterleaved {
    static __device__ __forceinline__ int2 load(const PlainParams &p, int i) {
        return __ldg(p.arcs + i);
    }
};
struct ArcsSplit {
    static __device__ __forceinline__ int2 load(const PlainParams &p, int i) {
        return make_int2(__ldg(p.col + i), __ldg(p.w + i));
    }
};

// Relaxes up to K rounds of 32 arcs whose destinations and candidate
// distances are known (round k: this lane's arc to dst[k] with candidate
// nd[k] when ok[k]) and feeds the winners to L1.  The rounds' destination-
// distance loads, then their updates, are issued back to back, so a warp
// keeps K independent chains in flight; `rounds` (warp-uniform) bounds the
// rounds that hold any arc.
template <int K>
__device__ __forceinline__ void relax_known(const PlainParams &p, WarpQ &q, uint2 *ring,
                                            const bool (&ok)[K], const unsigned (&dst)[K],
                                            const unsigned (&nd)[K], int rounds) {
    int cur[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
        cur[k] = INT_MAX;
        if (ok[k] && (p.precheck || nd[k] >= (unsigned)INT_MAX)) cur[k] = __ldcg(p.dist + dst[k]);
    }
    // With the pre-check the distance update is a fire-and-forget red.min and
    // the record is pushed when it beat the distance read: a push that a
    // concurrent smaller update made redundant is a stale record, which the
    // reader drops.  Without it, atomicMin's returned value decides.
    bool win[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
        win[k] = false;
        if (ok[k]) {
            if (nd[k] >= (unsigned)INT_MAX) {
                if (cur[k] == INT_MAX) {  // a finite distance would not fit
                    if constexpr (kStatsSmem) wstat()[WS_RANGE] = 1ull;
                    else q.range_hit = 1;
                }
            } else if ((int)nd[k] < cur[k]) {
                if (p.precheck) {
                    red_min(p.dist + dst[k], (int)nd[k]);
                    win[k] = true;
                } else {
                    win[k] = (int)nd[k] < atomicMin(p.dist + dst[k], (int)nd[k]);
                }
            }
        }
    }
    // Winners of all rounds are compacted into the warp's winner buffer and
    // go to L1 32 at a time: full warps, and one copy of the L1 code.
    const int lane = threadIdx.x & 31;
    uint2 *wb = ring + WINBUF_OFF;
    int nw = 0;
#pragma unroll
    for (int k = 0; k < K; k++) {
        if (k < rounds) {
            const unsigned m = __ballot_sync(FULL, win[k]);
            if (win[k]) wb[nw + (int)__popc(m & lanemask_lt())] = make_uint2(dst[k], nd[k]);
            nw += (int)__popc(m);
            if constexpr (!kStatsSmem) q.improved += win[k];
        }
    }
    if constexpr (kStatsSmem) wstat_add(WS_IMPROVED, (unsigned)nw);
    __syncwarp();
#pragma unroll 1
    for (int c = 0; c < nw; c += 32) {
        const bool ok = c + lane < nw;
        uint2 it = make_uint2(0u, 0u);
        if (ok) it = wb[c + lane];
        l1_write(p, q, ring, ok, it.x, it.y);
    }
    __syncwarp();
}

// Loads the arcs of K lane-distributed rounds (round k: this lane's arc ai[k]
// of a vertex at distance du[k] when ok[k]; a negative ai[k] is
// INT_MIN + an index into this warp's staged tile arcs), then relaxes them.
template <class Arcs, int K>
__device__ __forceinline__ void relax_rounds(const PlainParams &p, WarpQ &q, uint2 *ring,
                                             const int2 *stage, const bool (&ok)[K], const int (&ai)[K],
                                             const unsigned (&du)[K], int rounds) {
    unsigned dst[K], nd[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
        dst[k] = 0u;
        nd[k] = 0u;
        if (ok[k]) {
            const int2 a = ai[k] < 0 ? stage[(unsigned)ai[k] - 0x80000000u] : Arcs::load(p, ai[k]);
            dst[k] = (unsigned)a.x;
            nd[k] = du[k] + (unsigned)a.y;
        }
    }
    relax_known<K>(p, q, ring, ok, dst, nd, rounds);
}

// A heavy vertex is not relaxed by the warp that read it: one record per
// piece, at the vertex's distance, goes to L2, where any warp may take it.
// Lane-distributed as arcs are: an exclusive prefix sum of piece counts and
// a shuffle search for the owner lane of each piece.
__device__ __forceinline__ void push_pieces(const PlainParams &p, WarpQ &q, int np, int first,
                                            unsigned d) {
    const int lane = threadIdx.x & 31;
    int incl = np;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += t;
    }
    const int total = __shfl_sync(FULL, incl, 31);
    const int off = incl - np;
    for (int e0 = 0; e0 < total; e0 += 32) {
        const int e = e0 + lane;
        int j = 0;
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) {
            const int oc = __shfl_sync(FULL, off, j + s);
            if (oc <= e) j += s;
        }
        const int fj = __shfl_sync(FULL, first, j);
        const int oj = __shfl_sync(FULL, off, j);
        const unsigned dj = __shfl_sync(FULL, d, j);
        push32(p, q, e < total, (unsigned)(fj + (e - oj)), dj);
    }
}

// Relaxes up to 32 records (one per lane) and feeds the winners to L1.
// `stage` is this warp's TILE_ARCS_WIDE * 32 arcs of shared memory.
// kSplit: the graph may have split heavy vertices (pieces) or the
// light/heavy split may be on; a kernel built without them (graphs with no
// vertex above SPLIT_MIN arcs, light_heavy off) leaves their tests and code
// out -- a smaller loop body, fewer instruction-cache misses (C2 and C4 +5 %).
template <class Arcs, int K, bool kSplit>
__device__ __forceinline__ void relax_batch(const PlainParams &p, WarpQ &q, uint2 *ring,
                                            int2 *stage, bool valid, unsigned v, unsigned d) {
    const int lane = threadIdx.x & 31;
    int beg = 0, deg = 0;
    // Records are relaxed with their own distance: it is the length of a real
    // path, and with the fire-and-forget distance updates the update that
    // made the record may not be visible here yet.
    //
    // Light/heavy split (p.split non-null; delta-stepping's light and heavy
    // edges): arcs are sorted by weight, so a vertex's light arcs (w < delta)
    // are a prefix.  A fresh record relaxes the light arcs at once and pushes
    // one heavy record (id nslots + v) at distance + delta; heavy arcs cannot
    // improve anything in the record's own bucket, and when the heavy record
    // comes up the vertex's distance is (nearly always) final, so heavy arcs
    // are relaxed about once.  A heavy record is fresh while the vertex's
    // distance still equals the one it carries.
    const bool heavyrec = kSplit && valid && p.split && v >= (unsigned)p.nslots;
    if (heavyrec) {
        v -= (unsigned)p.nslots;
        d -= p.delta;
    }
    const unsigned du = d;
    if (p.tiles) {
        // Vertex tile: the distance (stale check) and the 32-byte tile are
        // independent loads.  A vertex of degree <= TILE_ARCS has all its arcs
        // in the tile: they are staged in shared memory and its `beg` becomes
        // INT_MIN + its stage offset, so the arc distribution below handles
        // staged and CSR arcs alike and keeps the CSR path's arc order.
        int cur = INT_MAX, light = 0;
        int4 ta = make_int4(-1, 0, -1, 0), tb = ta, tc = ta, td = ta;
        const bool piece = kSplit && valid && v >= (unsigned)p.n;
        const bool wide = p.tile_stride == 4;
        if (valid) {
            if (!piece) cur = __ldcg(p.dist + v);
            const int4 *t = p.tiles + (size_t)p.tile_stride * v;
            ta = __ldg(t);
            tb = __ldg(t + 1);
            if (wide) {
                tc = __ldg(t + 2);
                td = __ldg(t + 3);
            }
            if (kSplit && p.split && !piece) light = __ldg(p.split + v);
        }
        if (piece) cur = __ldcg(p.dist + ta.w);  // a piece is as fresh as its owner
        // Splitting needs room for distance + delta in a record.
        const bool lh = kSplit && p.split && !piece && d < (unsigned)INT_MAX - p.delta;
        int npieces = 0, first_piece = 0;
        bool push_heavy = false;
        if (valid && (int)d <= cur) {
            if (ta.x == TILE_CSR) {
                beg = ta.y;
                deg = ta.z;
                if (lh) {
                    if (heavyrec) {
                        beg += light;
                        deg -= light;
                    } else {
                        deg = light;
                        push_heavy = light < ta.z;
                    }
                }
            } else if (kSplit && ta.x == TILE_SPLIT) {
                first_piece = ta.y;
                npieces = ta.z;
                if (lh) {
                    // pieces are cut every PIECE_ARCS sorted arcs: the first
                    // nl hold every light arc
                    const int nl = (light + PIECE_ARCS - 1) / PIECE_ARCS;
                    if (heavyrec) {
                        first_piece += nl;
                        npieces -= nl;
                    } else {
                        npieces = nl;
                        push_heavy = nl < ta.z;
                    }
                }
            } else {
                int2 *st = stage + TILE_ARCS_WIDE * lane;
                st[0] = make_int2(ta.x, ta.y);
                st[1] = make_int2(ta.z, ta.w);
                st[2] = make_int2(tb.x, tb.y);
                st[3] = make_int2(tb.z, tb.w);
                int cnt = (ta.x >= 0) + (ta.z >= 0) + (tb.x >= 0) + (tb.z >= 0);
                if (wide) {
                    st[4] = make_int2(tc.x, tc.y);
                    st[5] = make_int2(tc.z, tc.w);
                    st[6] = make_int2(td.x, td.y);
                    st[7] = make_int2(td.z, td.w);
                    cnt += (tc.x >= 0) + (tc.z >= 0) + (td.x >= 0) + (td.z >= 0);
                }
                beg = INT_MIN + TILE_ARCS_WIDE * lane;
                deg = cnt;
                if (lh) {
                    // inline arcs are sorted by weight too
                    const unsigned dl = p.delta;
                    int nl = (cnt > 0 && (unsigned)ta.y < dl) + (cnt > 1 && (unsigned)ta.w < dl) +
                             (cnt > 2 && (unsigned)tb.y < dl) + (cnt > 3 && (unsigned)tb.w < dl);
                    if (wide)
                        nl += (cnt > 4 && (unsigned)tc.y < dl) + (cnt > 5 && (unsigned)tc.w < dl) +
                              (cnt > 6 && (unsigned)td.y < dl) + (cnt > 7 && (unsigned)td.w < dl);
                    if (heavyrec) {
                        beg += nl;
                        deg = cnt - nl;
                    } else {
                        deg = nl;
                        push_heavy = nl < cnt;
                    }
                }
            }
        }
        if (kSplit && __any_sync(FULL, npieces > 0)) push_pieces(p, q, npieces, first_piece, du);
        const unsigned hm = kSplit ? __ballot_sync(FULL, push_heavy) : 0u;
        if (hm) {
            // Heavy records wait in the outbox with the far winners and go
            // to L2 32 at a time: a push costs two L2 round trips whether it
            // carries 3 records or 32 (R-MAT-22 13.8 -> 14.5 GTEPS).  They
            // are a bucket ahead, and the outbox is empty before the warp
            // returns its read credit, so with bucket sync they reach L2
            // before the window moves past their bucket.
            if (push_heavy)
                ring[OUTBOX_OFF + q.ob_n + (int)__popc(hm & lanemask_lt())] =
                    make_uint2((unsigned)p.nslots + v, d + p.delta);
            __syncwarp();
            q.ob_n += (int)__popc(hm);
            if (q.ob_n >= 32) outbox_flush(p, q, ring, false);
        }
        __syncwarp();
    } else if (valid) {
        // The three loads are independent: issue them together rather than
        // after the stale check.
        const int cur = __ldcg(p.dist + v);
        const int rb = __ldg(p.row + v);
        const int re = __ldg(p.row + v + 1);
        if ((int)d <= cur) {
            beg = rb;
            deg = re - rb;
        }
    }
    if constexpr (kStatsSmem) wstat_add(WS_RELAXED, __reduce_add_sync(FULL, (unsigned)deg));
    else q.relaxed += (unsigned)deg;
    // Whole-warp relaxation of large vertices (sssp_run.cu:192-265).
    unsigned big = __ballot_sync(FULL, deg >= p.large);
    while (big) {
        const int sl = __ffs(big) - 1;
        big &= big - 1;
        const int lb = __shfl_sync(FULL, beg, sl);
        const int ld = __shfl_sync(FULL, deg, sl);
        const unsigned lu = __shfl_sync(FULL, du, sl);
        for (int e0 = 0; e0 < ld; e0 += 32 * K) {
            bool ok[K];
            int ai[K];
            unsigned uu[K];
#pragma unroll
            for (int k = 0; k < K; k++) {
                const int e = e0 + 32 * k + lane;
                ok[k] = e < ld;
                ai[k] = lb + e;
                uu[k] = lu;
            }
            relax_rounds<Arcs, K>(p, q, ring, stage, ok, ai, uu, (ld - e0 + 31) >> 5);
        }
    }
    if (deg >= p.large) deg = 0;
    // Small vertices: one arc per lane through an exclusive prefix sum of
    // degrees (sssp_run.cu:269-379); the owner lane of arc e is the last lane
    // whose offset is <= e, found by a 5-step shuffle search.
    int incl = deg;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += t;
    }
    const int total = __shfl_sync(FULL, incl, 31);
    const int off = incl - deg;
    if (K >= 4 && total <= 32) {
        // One round of arcs: the other rounds' owner searches and predicated
        // loads would be wasted on the critical path of a single solve.
        // (Measured: single solves 2.5-4 % faster; in the 2-round batched
        // instantiation the same branch cost 13 %, so only K = 4 has it.)
        if (total > 0) {
            int j = 0;
#pragma unroll
            for (int s = 16; s > 0; s >>= 1) {
                const int oc = __shfl_sync(FULL, off, j + s);
                if (oc <= lane) j += s;
            }
            const int ob = __shfl_sync(FULL, beg, j);
            const int oo = __shfl_sync(FULL, off, j);
            const bool ok1[1] = {lane < total};
            const int ai1[1] = {ob + (lane - oo)};
            const unsigned uu1[1] = {__shfl_sync(FULL, du, j)};
            relax_rounds<Arcs, 1>(p, q, ring, stage, ok1, ai1, uu1, 1);
        }
        return;
    }
    if (K >= 4 && total <= 64) {
        // Two rounds of arcs (C2: 2.35 -> 2.46 GTEPS over the one-round
        // dispatch alone).
        bool ok2[2];
        int ai2[2];
        unsigned uu2[2];
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const int e = 32 * k + lane;
            int j = 0;
#pragma unroll
            for (int s = 16; s > 0; s >>= 1) {
                const int oc = __shfl_sync(FULL, off, j + s);
                if (oc <= e) j += s;
            }
            const int ob = __shfl_sync(FULL, beg, j);
            const int oo = __shfl_sync(FULL, off, j);
            uu2[k] = __shfl_sync(FULL, du, j);
            ok2[k] = e < total;
            ai2[k] = ob + (e - oo);
        }
        relax_rounds<Arcs, 2>(p, q, ring, stage, ok2, ai2, uu2, 2);
        return;
    }
    for (int e0 = 0; e0 < total; e0 += 32 * K) {
        bool ok[K];
        int ai[K];
        unsigned uu[K];
#pragma unroll
        for (int k = 0; k < K; k++) {
            const int e = e0 + 32 * k + lane;
            int j = 0;
#pragma unroll
            for (int s = 16; s > 0; s >>= 1) {
                const int oc = __shfl_sync(FULL, off, j + s);
                if (oc <= e) j += s;
            }
            const int ob = __shfl_sync(FULL, beg, j);
            const int oo = __shfl_sync(FULL, off, j);
            uu[k] = __shfl_sync(FULL, du, j);
            ok[k] = e < total;
            ai[k] = ob + (e - oo);
        }
        relax_rounds<Arcs, K>(p, q, ring, stage, ok, ai, uu, (total - e0 + 31) >> 5);
    }
}

}  // namespace mlmq
