// device_common.cuh -- memory-model helpers, record encoding and the control
// block layout shared by the persistent delta-stepping kernels.
#pragma once

#include <climits>
#include <cstdint>
#include <cuda_runtime.h>

namespace mlmq {

constexpr unsigned FULL = 0xffffffffu;
constexpr int NB_MAX = 32;      // L2 buckets; lane b of a warp owns bucket b's claim
constexpr int L1_CAP = 64;      // SLF ring slots per warp (reference MAX_L1SLF_BATCH_SIZE)
constexpr unsigned long long SENT = ~0ull;  // empty ring slot
// Vertex tiles: 32 bytes per vertex, {dst, weight} x TILE_ARCS inline (unused
// slots dst = -1), or {TILE_CSR, first arc, degree, ...} for higher degree;
// wide tiles are 64 bytes with up to TILE_ARCS_WIDE arcs inline.
constexpr int TILE_ARCS = 4;
constexpr int TILE_ARCS_WIDE = 8;
constexpr int TILE_CSR = -2;
// A vertex of more than SPLIT_MIN arcs is relaxed as pieces of at most
// PIECE_ARCS arcs.  Piece k of the graph is a virtual vertex id n + k with
// tile {TILE_CSR, first arc, arcs, owner}; the heavy vertex's own tile is
// {TILE_SPLIT, first piece id, pieces, degree}.
constexpr int TILE_SPLIT = -3;
constexpr int SPLIT_MIN = 1024;
constexpr int PIECE_ARCS = 512;
// 8-byte shared-memory slots per worker warp: L1 ring, L2/L3 read buffer,
// staged tile arcs, outbox of records bound for L2/L3, winners of the
// relaxation rounds in flight (at most 4 rounds of 32).
constexpr int OUTBOX_CAP = 64;
constexpr int OUTBOX_OFF = L1_CAP + 32 + 32 * TILE_ARCS_WIDE;
constexpr int WINBUF_CAP = 128;
constexpr int WINBUF_OFF = OUTBOX_OFF + OUTBOX_CAP;
// Per-warp counters (u64) for kernels that keep them out of registers.
constexpr int WSTAT_OFF = WINBUF_OFF + WINBUF_CAP;
constexpr int WS_PUSHED = 0, WS_L3_PUSHED = 1, WS_RELAXED = 2, WS_IMPROVED = 3, WS_BATCHES = 4,
              WS_IDLE = 5, WS_RANGE = 6, WS_DEADLINE = 7;
constexpr int WARP_SMEM_SLOTS = WSTAT_OFF + 8;

// ---- control block: 32-bit words, one 128-byte line per group ------------
namespace ctl {
constexpr int FIRST = 0;      // current first bucket (absolute index)
constexpr int EXIT = 1;       // 1 = all warps leave the persistent loop
constexpr int STATUS = 2;     // ST_* bits
constexpr int PRESSURE = 3;   // bit b: L2 bucket b is filling, new pushes go to L3
constexpr int U_PRESSURE = 4; // 1: the urgent ring is filling, its pushes go to L3
constexpr int L3_MIN = 5;     // smallest distance pushed to L3 since the last L3 epoch
constexpr int L3_EPOCH = 6;   // L3 slots below this may be read (set when an epoch opens)
constexpr int BAR_COUNT = 8;  // grid barrier arrivals (self-resetting)
constexpr int BAR_GEN = 9;    // grid barrier generation
constexpr int CREDIT = 32;    // records read from L2/L3 whose work is finished
constexpr int RESERVE = 64;   // [NB_MAX] slots reserved per bucket
constexpr int CLAIM = 96;     // [NB_MAX] slots claimed by readers per bucket
constexpr int CONSUMED = 128; // [NB_MAX] slots read per bucket
constexpr int L3_RESERVE = 160;
constexpr int L3_CLAIM = 192;
constexpr int L3_CONSUMED = 224;
constexpr int STATS = 256;    // u64 counters (word offset, 8-byte aligned)
constexpr int ST_PUSHED = 0, ST_L3_PUSHED = 1, ST_RELAXED = 2, ST_IMPROVED = 3, ST_FIRST_MAX = 4,
              ST_BATCHES = 5, ST_IDLE = 6, ST_N = 8;
constexpr int WORDS = STATS + 2 * ST_N;  // 272 words
}  // namespace ctl

// status bits
constexpr unsigned ST_DONE = 1u;
constexpr unsigned ST_TIMEOUT = 2u;
constexpr unsigned ST_QUEUE_FULL = 4u;
constexpr unsigned ST_RANGE = 8u;
constexpr unsigned ST_SLOT_LOST = 16u;  // served query: its slot's CTAs could not meet

// ---- PTX memory-model helpers ------------------------------------------------
__device__ __forceinline__ unsigned ld_relaxed(const unsigned *p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(unsigned *p, unsigned v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_release(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed64(unsigned long long *p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
// atomicMin without a returned value: the issuing warp does not wait for it.
__device__ __forceinline__ void red_min(int *p, int v) {
    asm volatile("red.relaxed.gpu.global.min.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}
__device__ __forceinline__ unsigned lanemask_le() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_le;" : "=r"(m));
    return m;
}

// ---- queue records ---------------------------------------------------------
// One record is one 64-bit word: low half = vertex, high half = distance.
// Both are < 2^31, so bit 31 of each half is free; the two free bits carry the
// ring lap (slot index >> log2(capacity)) modulo 4.  A reader accepts a slot
// only when it holds a record of the lap it claimed, so a slot still holding
// the previous lap's record reads as "not yet written".  The all-ones word
// (SENT) is never a record: its vertex half would be 0x7fffffff >= n.
__device__ __forceinline__ unsigned long long rec_pack(unsigned v, unsigned d, unsigned lap) {
    const unsigned hi = d | (((lap >> 1) & 1u) << 31);
    const unsigned lo = v | ((lap & 1u) << 31);
    return ((unsigned long long)hi << 32) | (unsigned long long)lo;
}
__device__ __forceinline__ unsigned rec_lap(unsigned long long r) {
    return (((unsigned)r >> 31) & 1u) | (((unsigned)(r >> 62)) & 2u);
}
__device__ __forceinline__ unsigned rec_v(unsigned long long r) { return (unsigned)r & 0x7fffffffu; }
__device__ __forceinline__ unsigned rec_d(unsigned long long r) {
    return (unsigned)(r >> 32) & 0x7fffffffu;
}

// ---- result digest ---------------------------------------------------------
// A 64-bit fingerprint of a distance array: the sum, modulo 2^64, of
// mix64((v << 32) | dist[v]) over every vertex v, where mix64 is the
// SplitMix64 output function (Steele, Lea and Flood, 2014).  A sum of
// per-vertex terms, so any split of the vertices over threads gives the same
// value; mlmq_dist_digest computes it on the host.
__host__ __device__ __forceinline__ unsigned long long digest_mix64(unsigned long long x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
__host__ __device__ __forceinline__ unsigned long long digest_term(unsigned long long v, int d) {
    return digest_mix64((v << 32) | (unsigned)d);
}

// ---- grid barrier (the launch is cooperative, so every CTA is resident) ----
// Returns false when the wait ran past `deadline` (status gets ST_TIMEOUT).
__device__ __forceinline__ bool grid_barrier(unsigned *ctlw, unsigned nblocks,
                                             unsigned long long deadline) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        unsigned gen = ld_acquire(ctlw + ctl::BAR_GEN);
        __threadfence();
        unsigned arrived = atomicAdd(ctlw + ctl::BAR_COUNT, 1u);
        if (arrived == nblocks - 1) {
            st_relaxed(ctlw + ctl::BAR_COUNT, 0u);
            __threadfence();
            st_release(ctlw + ctl::BAR_GEN, gen + 1);
        } else {
            unsigned ns = 32;
            while (ld_acquire(ctlw + ctl::BAR_GEN) == gen) {
                if (globaltimer() > deadline) {
                    atomicOr(ctlw + ctl::STATUS, ST_TIMEOUT);
                    st_relaxed(ctlw + ctl::EXIT, 1u);
                    ok = 0;
                    break;
                }
                __nanosleep(ns);
                if (ns < 1024) ns <<= 1;
            }
        }
    }
    __syncthreads();
    return ok != 0;
}

}  // namespace mlmq
