// Greedy shared-mutation join of indel-coded cells on B200.
//
// Replaces cu/joinEdgeIndel.cu.  Same tree, same bytes; different machine
// mapping:
//
//  * Scores.  score(q, c) = sum over sites i with q_i == c_i and q_i > 1 of
//    w[(q_i-2)*ncol + i], accumulated in binary16 in ascending site order
//    (cu/joinEdgeIndel.cu:73-79).  When every binary16 weight is a
//    non-negative integer and the largest reachable sum is <= 2048, all
//    partial sums are exact, so an integer count (in packed 16-bit lanes)
//    gives identical values; otherwise the kernels add binary16 in site order
//    per candidate, as the reference does.
//  * Layout.  Cell codes live twice in HBM as u16: row-major by node (for
//    merges and output) and column-major by slot (site-major), so a query
//    reads only the columns of its own edited sites, 16 bytes (8 candidates)
//    per thread per site, fully coalesced.
//  * Initial local maxima (cu/joinEdgeIndel.cu:355-369) are one persistent
//    launch over (candidate chunk, query) tiles in chunk-major order: a 4096-
//    candidate chunk stays in L2 while every earlier query streams it, and the
//    per-query best is merged with a 64-bit atomicMax on (score, ~node) keys.
//  * The join loop (cu/joinEdgeIndel.cu:376-468) is one cooperative launch,
//    one CTA per SM, each owning a contiguous slot range.  Per join every CTA
//    redundantly derives the global best from the per-CTA records of the
//    previous phase, merges the two children, builds the query site list in
//    shared memory, scores its own slots and updates their local maxima; a
//    grid barrier (bounded wait) ends the phase.  A stale partner costs a
//    scoring phase plus an update phase, exactly like the reference's
//    recompute-and-retry.  Dead slots are squeezed out of the column matrix
//    whenever fewer than 3/4 of the slots are alive.
//  * Pre-order relabelling (cu/joinEdgeIndel.cu:488-558) walks the 2(N-1)
//    raw edges on the host in O(N) and gathers the state rows on device.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "runtime.h"

namespace casphy {
namespace indel {

constexpr int kThreads = 512;
constexpr int kG = 8;                       // candidates per thread (one uint4 of u16)
constexpr int kCap = kThreads * kG;         // candidates per pass
constexpr u32 kDead = 0xFFFFFFFFu;
constexpr u32 kNone = 0xFFFFFFFFu;
constexpr u32 kMaxCol = 16384;

struct BlockRec {
    u64 key;
    u32 slot;
    u32 partner;
};

__device__ __forceinline__ u32 half_bits_of_int(u32 s) { return __half_as_ushort(__uint2half_rn(s)); }

// Accumulate 8 candidates (cb .. cb+7 of column-major `col`, stride Sp) over
// the query entries e = e0, e0+step, ... < nE.  INT: packed 16-bit lane
// counts (acc[w] lanes = candidates 2w, 2w+1).  HALF: binary16 sums in order.
template <bool INTP>
struct Acc8;

template <>
struct Acc8<true> {
    u32 a[4];
    __device__ __forceinline__ void zero() { a[0] = a[1] = a[2] = a[3] = 0u; }
    __device__ __forceinline__ void add(const uint4 v, u32 qc, u32 w) {
        const u32 qq = qc * 0x00010001u;
        const u32 x[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int i = 0; i < 4; i++) {
            // lanes hold codes < 0x8000: a lane of t is zero iff it matches
            const u32 t = x[i] ^ qq;
            const u32 u = t + 0x7FFF7FFFu;
            const u32 m = (~u >> 15) & 0x00010001u;
            a[i] += m * w;
        }
    }
    __device__ __forceinline__ void store(u16* dst) const {
        *reinterpret_cast<uint4*>(dst) = make_uint4(a[0], a[1], a[2], a[3]);
    }
};

template <>
struct Acc8<false> {
    __half a[8];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int i = 0; i < 8; i++) a[i] = __ushort_as_half(0);
    }
    __device__ __forceinline__ void add(const uint4 v, u32 qc, u32 wbits) {
        const u32 x[4] = {v.x, v.y, v.z, v.w};
        const __half w = __ushort_as_half((u16)wbits);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            if ((x[i] & 0xFFFFu) == qc) a[2 * i] = __hadd(a[2 * i], w);
            if ((x[i] >> 16) == qc) a[2 * i + 1] = __hadd(a[2 * i + 1], w);
        }
    }
    __device__ __forceinline__ void store(u16* dst) const {
        u32 p[4];
#pragma unroll
        for (int i = 0; i < 4; i++)
            p[i] = (u32)__half_as_ushort(a[2 * i]) | ((u32)__half_as_ushort(a[2 * i + 1]) << 16);
        *reinterpret_cast<uint4*>(dst) = make_uint4(p[0], p[1], p[2], p[3]);
    }
};

template <bool INTP>
__device__ __forceinline__ void accumulate(Acc8<INTP>& acc, const u16* __restrict__ col, u32 Sp, u32 cb,
                                           const u32* eSC, const u16* eW, int e0, int nE, int step) {
    int e = e0;
    // eight independent 16-byte loads in flight per iteration
    for (; e + 7 * step < nE; e += 8 * step) {
        u32 sc[8], w[8];
        uint4 v[8];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            sc[i] = eSC[e + i * step];
            w[i] = eW[e + i * step];
        }
#pragma unroll
        for (int i = 0; i < 8; i++) v[i] = ld_cg_v4(col + (size_t)(sc[i] & 0xFFFFu) * Sp + cb);
#pragma unroll
        for (int i = 0; i < 8; i++) acc.add(v[i], sc[i] >> 16, w[i]);
    }
    for (; e < nE; e += step) {
        const u32 s0 = eSC[e];
        const uint4 v0 = ld_cg_v4(col + (size_t)(s0 & 0xFFFFu) * Sp + cb);
        acc.add(v0, s0 >> 16, eW[e]);
    }
}

// ---------------------------------------------------------------------------
// preparation kernels

struct PrepArgs {
    u32 ntip, ncol, ncolP, nState, Sp;
    const u32* codes;   // ntip x ncol
    const u16* Wsel;    // nState x ncol (int weights or binary16 bits)
    u32 maxCode;        // codes must be <= maxCode
    u16* nodeRow;       // nnode x ncolP
    u32* eSC;           // ntip x ncol
    u16* eW;            // ntip x ncol
    u32* eLen;          // ntip
    int* err;
};

// One warp per tip: narrow codes to u16, validate, and build the tip's
// ascending list of edited sites with their weights.
__global__ void k_prep_rows(PrepArgs a) {
    const u32 warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const u32 lane = threadIdx.x & 31;
    if (warp >= a.ntip) return;
    const u32* src = a.codes + (size_t)warp * a.ncol;
    u16* row = a.nodeRow + (size_t)warp * a.ncolP;
    u32* es = a.eSC + (size_t)warp * a.ncol;
    u16* ew = a.eW + (size_t)warp * a.ncol;
    u32 n = 0;
    for (u32 s0 = 0; s0 < a.ncolP; s0 += 32) {
        const u32 s = s0 + lane;
        u32 c = s < a.ncol ? src[s] : 0u;
        if (c > a.maxCode || (c > 1 && c - 2 >= a.nState)) {
            atomicCAS(a.err, 0, CASPHY_ERANGE);
            c = 0;
        }
        if (s < a.ncolP) row[s] = (u16)c;
        const bool ed = c > 1;
        const u32 bal = __ballot_sync(0xFFFFFFFFu, ed);
        if (ed) {
            const u32 pos = n + __popc(bal & ((1u << lane) - 1u));
            es[pos] = s | (c << 16);
            ew[pos] = a.Wsel[(size_t)(c - 2) * a.ncol + s];
        }
        n += __popc(bal);
    }
    if (lane == 0) a.eLen[warp] = n;
}

// colT[s][i] = nodeRow[i][s] for tips; padding slots [ntip, Sp) get code 0.
__global__ void k_transpose(const u16* __restrict__ nodeRow, u32 ntip, u32 ncol, u32 ncolP, u32 Sp,
                            u16* __restrict__ colT) {
    __shared__ u16 tile[32][33];
    const u32 i0 = blockIdx.x * 32, s0 = blockIdx.y * 32;
    for (u32 r = threadIdx.y; r < 32; r += blockDim.y) {
        const u32 i = i0 + r, s = s0 + threadIdx.x;
        tile[r][threadIdx.x] = (i < ntip && s < ncol) ? nodeRow[(size_t)i * ncolP + s] : (u16)0;
    }
    __syncthreads();
    for (u32 r = threadIdx.y; r < 32; r += blockDim.y) {
        const u32 s = s0 + r, i = i0 + threadIdx.x;
        if (s < ncol && i < Sp) colT[(size_t)s * Sp + i] = tile[threadIdx.x][r];
    }
}

// ---------------------------------------------------------------------------
// initial upper-triangle local maxima

struct InitArgs {
    u32 ntip, ncol, Sp;
    const u16* colT;
    const u32* eSC;
    const u16* eW;
    const u32* eLen;
    const u64* chunkStart;   // nChunks+1 prefix of tiles per chunk
    u32 nChunks;
    u64 nTiles;
    unsigned long long* tileCounter;
    unsigned long long* initKey;   // ntip
};

template <bool INTP>
__global__ void __launch_bounds__(kThreads) k_init_scan(InitArgs a) {
    __shared__ unsigned long long s_tile[2];
    __shared__ u64 red[32];
    if (threadIdx.x == 0) s_tile[0] = atomicAdd(a.tileCounter, 1ull);
    __syncthreads();
    int cur = 0;
    for (;;) {
        const u64 t = s_tile[cur];
        if (t >= a.nTiles) break;
        if (threadIdx.x == 0) s_tile[cur ^ 1] = atomicAdd(a.tileCounter, 1ull);
        u32 k = 0;
        while (k + 1 < a.nChunks && a.chunkStart[k + 1] <= t) k++;
        const u32 q = (u32)(t - a.chunkStart[k]);
        const u32 cb = k * kCap + threadIdx.x * kG;
        u64 best = make_key(ORD_F16_NEG1, 0u);
        if (cb < a.ntip && cb + kG > q + 1) {
            Acc8<INTP> acc;
            acc.zero();
            accumulate<INTP>(acc, a.colT, a.Sp, cb, a.eSC + (size_t)q * a.ncol, a.eW + (size_t)q * a.ncol, 0,
                             (int)a.eLen[q], 1);
            __align__(16) u16 v[8];
            acc.store(v);
#pragma unroll
            for (int m = 0; m < kG; m++) {
                const u32 j = cb + m;
                if (j > q && j < a.ntip) {
                    const u32 hb = INTP ? half_bits_of_int(v[m]) : v[m];
                    const u64 key = make_key(ord_f16((u16)hb), j);
                    best = key > best ? key : best;
                }
            }
        }
        best = block_max_u64(best, red);
        if (threadIdx.x == 0) atomicMax(a.initKey + q, (unsigned long long)best);
        cur ^= 1;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// persistent join loop

struct JoinArgs {
    u32 ntip, ncol, ncolP, nState, nnode, nCTA;
    u32 minSize;
    float minRatio;
    int unitW;
    const u16* Wsel;
    u16* nodeRow;
    u16* colT[2];
    u32* lmOrd[2];
    u32* lmIdx[2];
    u32* slotNode[2];
    u32* node2slot;
    u32* nodeDeath;
    u32* nodeSize;
    u32* rawEdge;
    BlockRec* pub;       // 2 phases x nCTA x 2 published records (best, second)
    u32* pubCnt;         // 2 phases x nCTA: live slots holding a real local max (capped at 3)
    u64* partial;        // 2 phases x nCTA
    u32* counts;         // nCTA
    u32* flags;          // nCTA x 16 barrier epochs
    int* err;
    u64 limitNs;
    unsigned long long* statsOut;  // [0] stale [1] pairs [2] compactions [3] phases [4] refreshes [5] alg bytes
    u32 Rmax;            // max slots per CTA (smem for compaction ranks)
};

struct Range {
    u32 S, Sp, R, lo, hi;
};

__device__ __forceinline__ Range make_range(u32 S, u32 nCTA, u32 b) {
    Range r;
    r.S = S;
    r.Sp = (S + 7u) & ~7u;
    u32 per = (S + nCTA - 1) / nCTA;
    r.R = (per + 7u) & ~7u;
    r.lo = min(b * r.R, S);
    r.hi = min(r.lo + r.R, S);
    return r;
}

// All-to-all flag barrier for a co-resident grid: CTA b publishes `epoch` in
// its own flag, threads 0..nCTA-1 each wait for one CTA's flag.  Every wait
// gives up after limit_ns and records CASPHY_ETIMEOUT.
__device__ __forceinline__ int flag_barrier(u32* flags, u32 nCTA, u32 epoch, int* err, u64 limit_ns) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        st_release_u32(flags + blockIdx.x * 16u, epoch);
    }
    int fail = 0;
    if (threadIdx.x < nCTA) {
        const u32* f = flags + threadIdx.x * 16u;
        if (ld_acquire_u32(f) < epoch) {
            const u64 t0 = globaltimer_ns();
            while (ld_acquire_u32(f) < epoch) {
                if (*(volatile int*)err) { fail = 1; break; }
                if (globaltimer_ns() - t0 > limit_ns) {
                    atomicCAS(err, 0, CASPHY_ETIMEOUT);
                    fail = 1;
                    break;
                }
                __nanosleep(40);
            }
        }
    }
    return __syncthreads_or(fail);
}

__device__ __forceinline__ u16* colT_of(const JoinArgs& a, u32 buf) { return buf ? a.colT[1] : a.colT[0]; }
__device__ __forceinline__ u32* lmOrd_of(const JoinArgs& a, u32 buf) { return buf ? a.lmOrd[1] : a.lmOrd[0]; }
__device__ __forceinline__ u32* lmIdx_of(const JoinArgs& a, u32 buf) { return buf ? a.lmIdx[1] : a.lmIdx[0]; }
__device__ __forceinline__ u32* slotNode_of(const JoinArgs& a, u32 buf) { return buf ? a.slotNode[1] : a.slotNode[0]; }

// Per-thread top-2 of (key, slot, partner) records.
struct Top2 {
    u64 k0, k1;
    u32 s0, s1, p0, p1;
    __device__ __forceinline__ void init() {
        k0 = k1 = 0ull;
        s0 = s1 = kNone;
        p0 = p1 = 0u;
    }
    __device__ __forceinline__ void push(u64 k, u32 s, u32 p) {
        if (k > k0) {
            k1 = k0; s1 = s0; p1 = p0;
            k0 = k; s0 = s; p0 = p;
        } else if (k > k1) {
            k1 = k; s1 = s; p1 = p;
        }
    }
};

// Block-wide argmax of records (keys are unique among live slots, so at most
// one thread holds the winner).
__device__ __forceinline__ BlockRec block_best_rec(u64 best, u32 bslot, u32 bpart, u64* red, BlockRec* s_rec) {
    if (threadIdx.x == 0) { s_rec->slot = kNone; s_rec->partner = 0; }
    const u64 m = block_max_u64(best, red);  // starts and ends with __syncthreads
    if (best == m && bslot != kNone && m != 0ull) { s_rec->slot = bslot; s_rec->partner = bpart; }
    __syncthreads();
    BlockRec r;
    r.key = m;
    r.slot = s_rec->slot;
    r.partner = s_rec->partner;
    __syncthreads();
    return r;
}

// Block top-2 from per-thread top-2 lists; returns them in out[0..1]
// (key 0 = absent).
__device__ __forceinline__ void block_top2(Top2 t, u64* red, BlockRec* s_rec, BlockRec* out) {
    BlockRec r0 = block_best_rec(t.k0, t.s0, t.p0, red, s_rec);
    if (t.k0 == r0.key && t.s0 == r0.slot && r0.key != 0ull) {
        t.k0 = t.k1; t.s0 = t.s1; t.p0 = t.p1;
        t.k1 = 0ull; t.s1 = kNone;
    }
    BlockRec r1 = block_best_rec(t.k0, t.s0, t.p0, red, s_rec);
    out[0] = r0;
    out[1] = r1;
}

// Publish this CTA's top-2 records and live-count for phase p.
__device__ __forceinline__ void publish(const JoinArgs& a, u32 p, u32 b, const BlockRec* top, u32 cnt) {
    if (threadIdx.x < 2) {
        BlockRec* dst = a.pub + ((size_t)(p & 1) * a.nCTA + b) * 2 + threadIdx.x;
        const BlockRec r = top[threadIdx.x];
        asm volatile("st.global.cg.v2.u64 [%0], {%1, %2};" ::"l"(dst), "l"(r.key),
                     "l"(((u64)r.partner << 32) | r.slot)
                     : "memory");
    }
    if (threadIdx.x == 2) a.pubCnt[(p & 1) * a.nCTA + b] = cnt;
}

// Local copy of every CTA's published top-2 list.  tab[2b], tab[2b+1];
// cnt[b] entries valid; exact[b]: the list holds every live slot of block b
// that carries a real local maximum.
struct Table {
    BlockRec* tab;
    unsigned char* cnt;
    unsigned char* exact;
};

__device__ void load_table(const JoinArgs& a, u32 p, Table t) {
    for (u32 i = threadIdx.x; i < a.nCTA * 2; i += kThreads) {
        const uint4 v = ld_cg_v4(a.pub + (size_t)(p & 1) * a.nCTA * 2 + i);
        BlockRec r;
        r.key = ((u64)v.y << 32) | v.x;
        r.slot = v.z;
        r.partner = v.w;
        t.tab[i] = r;
    }
    for (u32 i = threadIdx.x; i < a.nCTA; i += kThreads) {
        const u32 n = ld_cg_u32(a.pubCnt + (p & 1) * a.nCTA + i);
        t.cnt[i] = (unsigned char)min(n, 2u);
        t.exact[i] = n <= 2;
    }
    __syncthreads();
}

// Own top-2 straight from the stored local maxima (refresh / compaction).
__device__ void own_top2(const JoinArgs& a, u32 buf, const Range& rg, u64* red, BlockRec* s_rec, BlockRec* out,
                         u32* cntOut, u32* wsum) {
    Top2 t;
    t.init();
    u32 n = 0;
    const u32* sn = slotNode_of(a, buf);
    const u32* lo = lmOrd_of(a, buf);
    const u32* li = lmIdx_of(a, buf);
    for (u32 c = rg.lo + threadIdx.x; c < rg.hi; c += kThreads) {
        const u32 node = ld_cg_u32(sn + c);
        if (node == kDead) continue;
        const u32 o = ld_cg_u32(lo + c);
        if (o == ORD_F16_NEG1) continue;
        n++;
        t.push(make_key(o, node), c, ld_cg_u32(li + c));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xFFFFFFFFu, n, o);
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = n;
    block_top2(t, red, s_rec, out);  // contains __syncthreads
    u32 tot = 0;
    for (int w = 0; w < kThreads / 32; w++) tot += wsum[w];
    *cntOut = tot;
    __syncthreads();
}

// Builds the query site list (ascending sites with code > 1) from a row.
// mode 0: query = row1; 1: copy row2; 2: keep row1; 3: ancestral merge of
// row1 and row2 (updateAncestralKernel, cu/joinEdgeIndel.cu:87-99).  The row
// is also left in shared memory (mrow) for the write-back.
__device__ int build_query(const JoinArgs& a, const u16* row1, const u16* row2, int mode, u16* mrow, u32* eSC,
                           u16* eW, u32* wcount) {
    const u32 lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    // each thread owns a contiguous run of `per` sites so one block scan
    // keeps the list ascending
    const u32 per = (a.ncolP + kThreads - 1) / kThreads;
    const u32 s0 = threadIdx.x * per;
    u32 cnt = 0;
    u32 codes[4];
    const bool small = per <= 4;
    for (u32 i = 0; i < per; i++) {
        const u32 s = s0 + i;
        u32 c = 0;
        if (s < a.ncol) {
            const u32 x = ld_cg_u16(row1 + s);
            if (mode == 0 || mode == 2) {
                c = x;
            } else {
                const u32 y = ld_cg_u16(row2 + s);
                if (mode == 1) c = y;
                else c = (x == 0) ? y : ((y >= 1 && x != y) ? 1u : x);
            }
        }
        if (s < a.ncolP && mrow) mrow[s] = (u16)c;
        if (small) codes[i] = c;
        cnt += c > 1;
    }
    u32 incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const u32 n = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= (u32)o) incl += n;
    }
    if (lane == 31) wcount[wid] = incl;
    __syncthreads();
    if (threadIdx.x < 32) {
        const u32 v = threadIdx.x < kThreads / 32 ? wcount[threadIdx.x] : 0u;
        u32 wi = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const u32 n = __shfl_up_sync(0xFFFFFFFFu, wi, o);
            if (lane >= (u32)o) wi += n;
        }
        if (threadIdx.x < kThreads / 32) wcount[16 + threadIdx.x] = wi - v;
        if (threadIdx.x == 31) wcount[32] = wi;
    }
    __syncthreads();
    u32 pos = wcount[16 + wid] + incl - cnt;
    for (u32 i = 0; i < per; i++) {
        const u32 s = s0 + i;
        u32 c;
        if (small) c = codes[i];
        else c = s < a.ncolP && mrow ? mrow[s] : (s < a.ncol ? ld_cg_u16(row1 + s) : 0u);
        if (c > 1) {
            eSC[pos] = s | (c << 16);
            eW[pos] = a.unitW ? (u16)1 : a.Wsel[(size_t)(c - 2) * a.ncol + s];
            pos++;
        }
    }
    const int n = (int)wcount[32];
    __syncthreads();
    return n;
}

// Scores this CTA's live slots against the query list.
// STALE: returns (in top[0]) the best (score, node) over slots != c1.
// JOIN: updates local maxima (strict improvement, cu/joinEdgeIndel.cu:453-460)
// and returns the CTA's top-2 records; *cntOut = slots with a real maximum.
template <bool INTP, bool JOIN>
__device__ void scan_own(const JoinArgs& a, u32 buf, const Range& rg, int nE, const u32* eSC, const u16* eW,
                         u16* part, u32 c1, u32 newNode, u64* red, BlockRec* s_rec, BlockRec* top, u32* cntOut,
                         u32* wsum) {
    const u32 R = rg.hi - rg.lo;
    int F = 1;
    if (INTP) {
        while (F < 16 && (u32)(kCap / (F * 2)) >= R) F *= 2;
    }
    const u32 cap = kCap / F;
    const u32 Tg = kThreads / F;
    const u32 g = threadIdx.x / Tg, t = threadIdx.x % Tg;
    Top2 tt;
    tt.init();
    u32 n = 0;
    const u32* sn = slotNode_of(a, buf);
    u32* lop = lmOrd_of(a, buf);
    u32* lip = lmIdx_of(a, buf);
    for (u32 base = rg.lo; base < rg.hi; base += cap) {
        const u32 cb = base + t * kG;
        Acc8<INTP> acc;
        acc.zero();
        if (cb < rg.hi) accumulate<INTP>(acc, colT_of(a, buf), rg.Sp, cb, eSC, eW, (int)g, nE, F);
        acc.store(part + g * cap + t * kG);
        __syncthreads();
        for (u32 x = threadIdx.x; x < cap; x += kThreads) {
            const u32 c = base + x;
            if (c >= rg.hi) break;
            const u32 node = ld_cg_u32(sn + c);
            if (node == kDead || c == c1) continue;
            u32 hb;
            if (INTP) {
                u32 sum = 0;
                for (int gg = 0; gg < F; gg++) sum += part[gg * cap + x];
                hb = half_bits_of_int(sum);
            } else {
                hb = part[x];
            }
            const u32 o = ord_f16((u16)hb);
            if (JOIN) {
                u32 lo = ld_cg_u32(lop + c);
                u32 li;
                if (o > lo) {
                    lo = o;
                    li = newNode;
                    lop[c] = o;
                    lip[c] = newNode;
                } else {
                    li = ld_cg_u32(lip + c);
                }
                if (lo != ORD_F16_NEG1) {
                    n++;
                    tt.push(make_key(lo, node), c, li);
                }
            } else {
                tt.push(make_key(o, node), c, 0u);
            }
        }
        __syncthreads();
    }
    if (JOIN) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xFFFFFFFFu, n, o);
        if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = n;
        block_top2(tt, red, s_rec, top);
        u32 tot = 0;
        for (int w = 0; w < kThreads / 32; w++) tot += wsum[w];
        *cntOut = tot;
        __syncthreads();
    } else {
        top[0] = block_best_rec(tt.k0, tt.s0, 0u, red, s_rec);
    }
}

// Decision shared by every CTA: the best published record over all blocks.
// Returns false when a block's best is unknown (its list was used up by
// stale updates) so the owners must republish first.
__device__ bool table_best(const Table& t, u32 nCTA, BlockRec* s_best, u64* red) {
    __shared__ int s_unknown;
    if (threadIdx.x == 0) s_unknown = 0;
    __syncthreads();
    u64 best = 0ull;
    u32 bi = kNone;
    for (u32 i = threadIdx.x; i < nCTA; i += kThreads) {
        if (t.cnt[i] == 0) {
            if (!t.exact[i]) s_unknown = 1;
            continue;
        }
        if (t.tab[2 * i].key > best) { best = t.tab[2 * i].key; bi = i; }
    }
    const u64 m = block_max_u64(best, red);
    if (best == m && bi != kNone) *s_best = t.tab[2 * bi];
    __syncthreads();
    const bool ok = s_unknown == 0 && m != 0ull;
    return ok;
}

template <bool INTP>
__global__ void __launch_bounds__(kThreads, 1) k_join(JoinArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    u16* part = reinterpret_cast<u16*>(smem);                          // kCap u16
    BlockRec* tabRec = reinterpret_cast<BlockRec*>(part + kCap);       // 2*nCTA
    u32* eSC = reinterpret_cast<u32*>(tabRec + 2 * a.nCTA);            // ncol
    u32* ranks = eSC + a.ncol;                                         // Rmax
    u16* eW = reinterpret_cast<u16*>(ranks + a.Rmax);                  // ncol (rounded to 8)
    u16* mrow = eW + ((a.ncol + 7u) & ~7u);                            // ncolP
    unsigned char* tabCnt = reinterpret_cast<unsigned char*>(mrow + a.ncolP);  // nCTA
    unsigned char* tabExact = tabCnt + a.nCTA;                         // nCTA
    __shared__ u64 red[32];
    __shared__ BlockRec s_rec, s_best;
    __shared__ BlockRec s_top[2];
    __shared__ u32 wcount[40];
    __shared__ u32 wsum[16];
    __shared__ u32 s_val[4];

    const Table T{tabRec, tabCnt, tabExact};
    const u32 b = blockIdx.x, nCTA = a.nCTA;
    u32 buf = 0;
    Range rg = make_range(a.ntip, nCTA, b);
    u32 k = 0, p = 0;
    unsigned long long nStale = 0, nPairs = 0, nComp = 0, nRefresh = 0, algBytes = 0;
    const u32 nJoin = a.ntip - 1;
    int fail = 0;
    u32 cnt = 0;

    own_top2(a, buf, rg, red, &s_rec, s_top, &cnt, wsum);
    publish(a, p, b, s_top, cnt);
    if (flag_barrier(a.flags, nCTA, ++p, a.err, a.limitNs)) goto out;
    load_table(a, p - 1, T);

    while (k < nJoin) {
        if (!table_best(T, nCTA, &s_best, red)) {
            // a block's best is unknown: every CTA republishes from its slots
            own_top2(a, buf, rg, red, &s_rec, s_top, &cnt, wsum);
            publish(a, p, b, s_top, cnt);
            nRefresh++;
            if (flag_barrier(a.flags, nCTA, ++p, a.err, a.limitNs)) goto out;
            load_table(a, p - 1, T);
            continue;
        }
        const BlockRec g = s_best;
        const u32 j1 = key_node(g.key), c1 = g.slot, j2 = g.partner;
        if (c1 >= rg.S || j1 >= a.nnode || j2 >= a.nnode) { fail = CASPHY_EINTERNAL; break; }
        if (threadIdx.x == 0) {
            s_val[0] = ld_cg_u32(a.nodeDeath + j2);
            s_val[1] = ld_cg_u32(a.node2slot + j2);
            s_val[2] = ld_cg_u32(a.nodeSize + j1);
            s_val[3] = ld_cg_u32(a.nodeSize + j2);
        }
        __syncthreads();
        const u32 death = s_val[0], c2 = s_val[1], s1 = s_val[2], s2 = s_val[3];
        __syncthreads();
        const bool stale = death < k || c2 >= rg.S;
        if (stale) {
            // rescore j1 against every live slot (cu/joinEdgeIndel.cu:387-399)
            const int nE = build_query(a, a.nodeRow + (size_t)j1 * a.ncolP, nullptr, 0, nullptr, eSC, eW, wcount);
            scan_own<INTP, false>(a, buf, rg, nE, eSC, eW, part, c1, 0u, red, &s_rec, s_top, nullptr, wsum);
            if (threadIdx.x == 0) {
                asm volatile("st.global.cg.u64 [%0], %1;" ::"l"(a.partial + (p & 1) * nCTA + b), "l"(s_top[0].key)
                             : "memory");
            }
            nStale++;
            nPairs += (a.ntip - k) - 1;
            algBytes += 2ull * (u64)nE * ((a.ntip - k) - 1);
            if (flag_barrier(a.flags, nCTA, ++p, a.err, a.limitNs)) goto out;
            u64 pb = make_key(ORD_F16_NEG1, 0u);
            for (u32 i = threadIdx.x; i < nCTA; i += kThreads) {
                const u64 v = ld_cg_u64(a.partial + ((p - 1) & 1) * nCTA + i);
                pb = v > pb ? v : pb;
            }
            pb = block_max_u64(pb, red);
            const u32 vOrd = key_ord(pb), vIdx = key_node(pb);
            const u32 ob = c1 / rg.R;  // owner CTA of c1
            if (ob == b && threadIdx.x == 0) {
                lmOrd_of(a, buf)[c1] = vOrd;
                lmIdx_of(a, buf)[c1] = vIdx;
            }
            // replace c1's entry (the head of its owner's list) in the table
            if (threadIdx.x == 0) {
                BlockRec nr;
                nr.key = make_key(vOrd, j1);
                nr.slot = c1;
                nr.partner = vIdx;
                BlockRec* L = T.tab + 2 * ob;
                unsigned char n = T.cnt[ob];
                // drop the head (c1)
                if (n == 2) L[0] = L[1];
                n = n > 0 ? n - 1 : 0;
                const bool real = vOrd != ORD_F16_NEG1;
                if (T.exact[ob]) {
                    if (real) {
                        if (n == 0) L[0] = nr;
                        else if (nr.key > L[0].key) { L[1] = L[0]; L[0] = nr; }
                        else L[1] = nr;
                        n++;
                    }
                    if (n > 2) n = 2;
                } else if (n >= 1 && real && nr.key > L[n - 1].key) {
                    if (nr.key > L[0].key) { L[1] = L[0]; L[0] = nr; }
                    else L[1] = nr;
                    n = 2;
                }
                T.cnt[ob] = n;
            }
            __syncthreads();
            continue;
        }
        // join j1 and j2 into node ntip+k (cu/joinEdgeIndel.cu:402-467)
        const u32 newNode = a.ntip + k;
        int mode;
        if (s1 < a.minSize && __uint2float_rn(s1) * a.minRatio < __uint2float_rn(s2)) mode = 1;
        else if (s2 < a.minSize && __uint2float_rn(s2) * a.minRatio < __uint2float_rn(s1)) mode = 2;
        else mode = 3;
        const int nE = build_query(a, a.nodeRow + (size_t)j1 * a.ncolP, a.nodeRow + (size_t)j2 * a.ncolP, mode, mrow,
                                   eSC, eW, wcount);
        if (b == 0) {
            u16* dst = a.nodeRow + (size_t)newNode * a.ncolP;
            for (u32 s = threadIdx.x; s < a.ncolP; s += kThreads) dst[s] = mrow[s];
            if (threadIdx.x == 0) {
                a.nodeSize[newNode] = s1 + s2;
                a.rawEdge[4 * k + 0] = newNode;
                a.rawEdge[4 * k + 1] = j1;
                a.rawEdge[4 * k + 2] = newNode;
                a.rawEdge[4 * k + 3] = j2;
                a.node2slot[newNode] = c1;
                a.nodeDeath[j1] = k;
                a.nodeDeath[j2] = k;
            }
        }
        if (c1 >= rg.lo && c1 < rg.hi) {
            u16* col = colT_of(a, buf);
            for (u32 s = threadIdx.x; s < a.ncol; s += kThreads) col[(size_t)s * rg.Sp + c1] = mrow[s];
            if (threadIdx.x == 0) {
                slotNode_of(a, buf)[c1] = newNode;
                lmOrd_of(a, buf)[c1] = ORD_F16_NEG1;
            }
        }
        if (c2 >= rg.lo && c2 < rg.hi && threadIdx.x == 0) {
            slotNode_of(a, buf)[c2] = kDead;
            lmOrd_of(a, buf)[c2] = ORD_F16_NEG1;
        }
        __syncthreads();
        scan_own<INTP, true>(a, buf, rg, nE, eSC, eW, part, c1, newNode, red, &s_rec, s_top, &cnt, wsum);
        publish(a, p, b, s_top, cnt);
        nPairs += (a.ntip - k - 1) - 1;
        algBytes += 2ull * (u64)nE * ((a.ntip - k - 1) - 1);
        k++;
        if (flag_barrier(a.flags, nCTA, ++p, a.err, a.limitNs)) goto out;
        load_table(a, p - 1, T);

        // squeeze dead slots out when fewer than 3/4 are alive
        const u32 alive = a.ntip - k;
        if (k < nJoin && rg.S >= 4096 && (u64)alive * 4 < (u64)rg.S * 3) {
            // C1: live slots per CTA
            const u32* sn = slotNode_of(a, buf);
            {
                u32 v = 0;
                for (u32 c = rg.lo + threadIdx.x; c < rg.hi; c += kThreads) v += ld_cg_u32(sn + c) != kDead;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
                if ((threadIdx.x & 31) == 0) wcount[threadIdx.x >> 5] = v;
                __syncthreads();
                if (threadIdx.x == 0) {
                    u32 tot = 0;
                    for (int w = 0; w < kThreads / 32; w++) tot += wcount[w];
                    a.counts[b] = tot;
                }
                __syncthreads();
            }
            if (flag_barrier(a.flags, nCTA, ++p, a.err, a.limitNs)) goto out;
            // C2: new positions = exclusive prefix of the per-CTA live counts
            if (threadIdx.x == 0) {
                u32 off = 0, tot = 0;
                for (u32 i = 0; i < nCTA; i++) {
                    const u32 v = ld_cg_u32(a.counts + i);
                    if (i < b) off += v;
                    tot += v;
                }
                s_val[0] = off;
                s_val[1] = tot;
            }
            __syncthreads();
            const u32 off = s_val[0], Snew = s_val[1];
            __syncthreads();
            if (Snew != alive) { fail = CASPHY_EINTERNAL; break; }
            const u32 Spn = (Snew + 7u) & ~7u;
            const u32 nb = buf ^ 1u;
            u32* snN = slotNode_of(a, nb);
            u32* loN = lmOrd_of(a, nb);
            u32* liN = lmIdx_of(a, nb);
            {
                const u32 R = rg.hi - rg.lo;
                const u32 per = (R + kThreads - 1) / kThreads;
                const u32 c0 = rg.lo + threadIdx.x * per;
                const u32 cEnd = min(c0 + per, rg.hi);
                u32 v = 0;
                for (u32 c = c0; c < cEnd; c++) v += ld_cg_u32(sn + c) != kDead;
                u32 incl = v;
                const u32 lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    u32 nn = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                    if (lane >= (u32)o) incl += nn;
                }
                if (lane == 31) wcount[wid] = incl;
                __syncthreads();
                if (threadIdx.x < 32) {
                    u32 wv = threadIdx.x < kThreads / 32 ? wcount[threadIdx.x] : 0u, wi = wv;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        u32 nn = __shfl_up_sync(0xFFFFFFFFu, wi, o);
                        if (lane >= (u32)o) wi += nn;
                    }
                    if (threadIdx.x < kThreads / 32) wcount[16 + threadIdx.x] = wi - wv;
                }
                __syncthreads();
                u32 r = off + wcount[16 + wid] + incl - v;
                const u32* lo = lmOrd_of(a, buf);
                const u32* li = lmIdx_of(a, buf);
                for (u32 c = c0; c < cEnd; c++) {
                    const u32 node = ld_cg_u32(sn + c);
                    if (node != kDead) {
                        ranks[c - rg.lo] = r;
                        snN[r] = node;
                        loN[r] = ld_cg_u32(lo + c);
                        liN[r] = ld_cg_u32(li + c);
                        a.node2slot[node] = r;
                        r++;
                    } else {
                        ranks[c - rg.lo] = kNone;
                    }
                }
                __syncthreads();
                const u16* src = colT_of(a, buf);
                u16* dst = colT_of(a, nb);
                for (u32 s = 0; s < a.ncol; s++) {
                    for (u32 x = threadIdx.x; x < R; x += kThreads) {
                        const u32 rr = ranks[x];
                        if (rr != kNone) dst[(size_t)s * Spn + rr] = ld_cg_u16(src + (size_t)s * rg.Sp + rg.lo + x);
                    }
                }
            }
            if (b == 0 && threadIdx.x < Spn - Snew) {
                snN[Snew + threadIdx.x] = kDead;
                loN[Snew + threadIdx.x] = ORD_F16_NEG1;
            }
            if (flag_barrier(a.flags, nCTA, ++p, a.err, a.limitNs)) goto out;
            // C3: switch to the compacted buffers and republish
            buf = nb;
            rg = make_range(Snew, nCTA, b);
            own_top2(a, buf, rg, red, &s_rec, s_top, &cnt, wsum);
            publish(a, p, b, s_top, cnt);
            nComp++;
            if (flag_barrier(a.flags, nCTA, ++p, a.err, a.limitNs)) goto out;
            load_table(a, p - 1, T);
        }
    }
out:
    if (fail && threadIdx.x == 0) atomicCAS(a.err, 0, fail);
    if (b == 0 && threadIdx.x == 0) {
        a.statsOut[0] = nStale;
        a.statsOut[1] = nPairs;
        a.statsOut[2] = nComp;
        a.statsOut[3] = p;
        a.statsOut[4] = nRefresh;
        a.statsOut[5] = algBytes;
    }
}

// state_out[r] = nodeRow[order[r]] widened to u32
__global__ void k_gather(const u16* __restrict__ nodeRow, u32 ncol, u32 ncolP, const u32* __restrict__ order, u32 nrows,
                         u32* __restrict__ out) {
    const u32 r = blockIdx.x;
    if (r >= nrows) return;
    const u16* src = nodeRow + (size_t)order[r] * ncolP;
    u32* dst = out + (size_t)r * ncol;
    for (u32 s = threadIdx.x; s < ncol; s += blockDim.x) dst[s] = src[s];
}

__global__ void k_slot_init(u32 ntip, u32 Sp, u32 nnode, const unsigned long long* initKey, u32* lmOrd, u32* lmIdx,
                            u32* slotNode, u32* node2slot, u32* nodeDeath, u32* nodeSize, const u32* tipSize) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < Sp) {
        if (i < ntip) {
            const u64 k = initKey[i];
            lmOrd[i] = key_ord(k);
            lmIdx[i] = key_node(k);
            slotNode[i] = i;
        } else {
            lmOrd[i] = ORD_F16_NEG1;
            lmIdx[i] = 0;
            slotNode[i] = kDead;
        }
    }
    if (i < nnode) {
        node2slot[i] = i < ntip ? i : kNone;
        nodeDeath[i] = kNone;
        nodeSize[i] = i < ntip ? tipSize[i] : 0u;
    }
}

__global__ void k_fill_u64(unsigned long long* p, u64 n, u64 v) {
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

}  // namespace indel

// ---------------------------------------------------------------------------
// host side

using namespace indel;

// Pre-order walk of the raw join edges (cu/joinEdgeIndel.cu:488-558): node v's
// edges are 2(v-ntip) (first child) and 2(v-ntip)+1; the root is 2ntip-2.
// Writes the relabelled edge list and the node id of every state row.
void preorder_relabel(u32 ntip, const u32* rawEdge, u32* edge_out, std::vector<u32>& order) {
    const u32 nnode = 2 * ntip - 1, nedge = 2 * ntip - 2;
    std::vector<u32> relabel(nnode);
    for (u32 i = 0; i < nnode; i++) relabel[i] = i < ntip ? i : nnode;
    std::vector<u32> stack;
    std::vector<unsigned char> cursor(nnode, 0);
    stack.reserve(nnode);
    order.clear();
    order.reserve(ntip);
    order.push_back(nnode - 1);
    stack.push_back(nnode - 1);
    u32 count = ntip, nout = 0;
    while (!stack.empty()) {
        const u32 v = stack.back();
        if (v < ntip || cursor[v] >= 2) { stack.pop_back(); continue; }
        const u32 ei = 2 * (v - ntip) + cursor[v];
        cursor[v]++;
        const u32 p = rawEdge[2 * ei], c = rawEdge[2 * ei + 1];
        stack.push_back(c);
        if (relabel[p] == nnode) relabel[p] = count++;
        if (relabel[c] == nnode) {
            order.push_back(c);
            relabel[c] = count++;
        }
        edge_out[2 * nout] = relabel[p];
        edge_out[2 * nout + 1] = relabel[c];
        nout++;
    }
    (void)nedge;
}

// binary16 conversion of the weight table, and the exactness test for the
// integer path: every weight a non-negative integer and the largest reachable
// score (sum over sites of the site's largest weight) at most 2048.
static int convert_weights(u32 nState, u32 ncol, const double* w, std::vector<u16>& hbits, std::vector<u16>& wint,
                           bool& intPath, bool& unitW) {
    const size_t n = (size_t)nState * ncol;
    hbits.resize(n ? n : 1);
    wint.resize(n ? n : 1);
    intPath = true;
    unitW = true;
    double maxSum = 0;
    std::vector<double> colMax(ncol, 0.0);
    for (size_t i = 0; i < n; i++) {
        const double x = w[i];
        if (std::isnan(x) || x < 0) {
            casphy_set_last_error_msg("weights must be >= 0 and not NaN");
            return CASPHY_EINVAL;
        }
        const __half h = __double2half(x);
        const u16 hb = __half_as_ushort(h);
        hbits[i] = hb;
        const float hf = __half2float(h);
        if (!(hf == std::floor(hf) && hf <= 2048.0f)) intPath = false;
        wint[i] = intPath ? (u16)hf : 0;
        if (hf != 1.0f) unitW = false;
        colMax[i % ncol] = std::max(colMax[i % ncol], (double)hf);
    }
    for (u32 i = 0; i < ncol; i++) maxSum += colMax[i];
    if (maxSum > 2048.0) intPath = false;
    if ((u64)nState + 1 > 0x7FFFu) intPath = false;  // packed-lane compare needs codes < 0x8000
    if (!intPath) unitW = false;
    return CASPHY_OK;
}

static int join_indel_impl(u32 ntip, u32 ncol, const u32* d_codes, u32 nState, const double* weight,
                           const u32* tipSize, u32 minSize, float minRatio, u32* edge_out, u32* d_state_out,
                           u32* h_state_out, casphy_join_stats* stats, cudaStream_t st, DeviceScope& ds,
                           const u32* h_codes) {
    if (ntip == 0 || ncol == 0 || !weight || !tipSize || !edge_out) return CASPHY_EINVAL;
    if (ncol > kMaxCol) {
        casphy_set_last_error_msg("ncol exceeds 16384");
        return CASPHY_ERANGE;
    }
    std::vector<u16> hbits, wint;
    bool intPath = false, unitW = false;
    int rc = convert_weights(nState, ncol, weight, hbits, wint, intPath, unitW);
    if (rc) return rc;
    casphy_join_stats lst{};
    lst.int_path = intPath ? 1 : 0;
    const u32 nnode = 2 * ntip - 1, nedge = 2 * ntip - 2;
    const u32 ncolP = (ncol + 7u) & ~7u;
    const u32 Sp = (ntip + 7u) & ~7u;
    int dev = ds.dev, nSM = 0;
    CASPHY_CUDA_TRY(cudaDeviceGetAttribute(&nSM, cudaDevAttrMultiProcessorCount, dev));

    const u32 nCTA = (u32)nSM;
    const u32 Rmax = (((ntip + nCTA - 1) / nCTA) + 7u) & ~7u;
    // device layout
    Carve cv;
    auto layout = [&](Carve& c) {
        struct L {
            u32* codes; u16* Wsel; u16* nodeRow; u16* colT0; u16* colT1; u32* lm[6];
            u32* node2slot; u32* nodeDeath; u32* nodeSize; u32* rawEdge; u32* eSC; u16* eW; u32* eLen;
            unsigned long long* initKey; BlockRec* pub; u32* pubCnt; u64* partial; u32* counts; u32* flags; int* jerr;
            unsigned long long* tileCounter; u64* chunkStart; unsigned long long* stats; u32* order; u32* tipSize;
            u32* stateOut; int* err;
        } l;
        l.codes = c.take<u32>(h_codes ? (size_t)ntip * ncol : 0);
        l.Wsel = c.take<u16>(hbits.size());
        l.nodeRow = c.take<u16>((size_t)nnode * ncolP);
        l.colT0 = c.take<u16>((size_t)ncol * Sp);
        l.colT1 = c.take<u16>((size_t)ncol * Sp);
        for (int i = 0; i < 6; i++) l.lm[i] = c.take<u32>(Sp);
        l.node2slot = c.take<u32>(nnode);
        l.nodeDeath = c.take<u32>(nnode);
        l.nodeSize = c.take<u32>(nnode);
        l.rawEdge = c.take<u32>((size_t)2 * nedge + 2);
        l.eSC = c.take<u32>((size_t)ntip * ncol);
        l.eW = c.take<u16>((size_t)ntip * ncol);
        l.eLen = c.take<u32>(ntip);
        l.initKey = c.take<unsigned long long>(ntip);
        l.pub = c.take<BlockRec>(4 * nCTA);
        l.pubCnt = c.take<u32>(2 * nCTA);
        l.partial = c.take<u64>(2 * nCTA);
        l.counts = c.take<u32>(nCTA);
        l.flags = c.take<u32>(16 * nCTA);
        l.jerr = c.take<int>(1);
        l.tileCounter = c.take<unsigned long long>(1);
        l.chunkStart = c.take<u64>(1024);
        l.stats = c.take<unsigned long long>(8);
        l.order = c.take<u32>(ntip);
        l.tipSize = c.take<u32>(ntip);
        l.stateOut = c.take<u32>(h_state_out ? (size_t)std::max(ntip - 1, 1u) * ncol : 0);
        l.err = c.take<int>(1);
        return l;
    };
    layout(cv);
    void* base = nullptr;
    rc = ds.reserve(cv.off + 256, &base);
    if (rc) return rc;
    Carve c2;
    c2.base = static_cast<char*>(base);
    auto L = layout(c2);
    const u32* codes = d_codes;
    if (h_codes) {
        CASPHY_CUDA_TRY(cudaMemcpyAsync(L.codes, h_codes, sizeof(u32) * (size_t)ntip * ncol, cudaMemcpyHostToDevice, st));
        codes = L.codes;
    }
    cudaEvent_t ev[6];
    for (auto& e : ev) CASPHY_CUDA_TRY(cudaEventCreate(&e));
    CASPHY_CUDA_TRY(cudaEventRecord(ev[0], st));
    CASPHY_CUDA_TRY(cudaMemcpyAsync(L.Wsel, intPath ? wint.data() : hbits.data(), sizeof(u16) * hbits.size(),
                                    cudaMemcpyHostToDevice, st));
    CASPHY_CUDA_TRY(cudaMemcpyAsync(L.tipSize, tipSize, sizeof(u32) * ntip, cudaMemcpyHostToDevice, st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(L.err, 0, sizeof(int), st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(L.flags, 0, sizeof(u32) * 16 * nCTA, st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(L.jerr, 0, sizeof(int), st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(L.tileCounter, 0, sizeof(unsigned long long), st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(L.stats, 0, sizeof(unsigned long long) * 8, st));
    u64 launches = 0;

    PrepArgs pa{ntip, ncol, ncolP, nState, Sp, codes, L.Wsel, intPath ? 0x7FFFu : 0xFFFFu,
                L.nodeRow, L.eSC, L.eW, L.eLen, L.err};
    k_prep_rows<<<(ntip + 7) / 8, 256, 0, st>>>(pa);
    dim3 tg((Sp + 31) / 32, (ncol + 31) / 32);
    k_transpose<<<tg, dim3(32, 8), 0, st>>>(L.nodeRow, ntip, ncol, ncolP, Sp, L.colT0);
    launches += 2;
    // tiles: chunk k holds candidates [k*kCap, (k+1)*kCap); queries i < min(end, ntip) - 1
    const u32 nChunks = (ntip + kCap - 1) / kCap;
    if (nChunks + 1 > 1024) {
        casphy_set_last_error_msg("too many cells for the chunk table");
        return CASPHY_ERANGE;
    }
    std::vector<u64> chunkStart(nChunks + 1, 0);
    for (u32 k = 0; k < nChunks; k++) {
        const u64 end = std::min<u64>((u64)(k + 1) * kCap, ntip);
        chunkStart[k + 1] = chunkStart[k] + (end >= 1 ? end - 1 : 0);
    }
    const u64 nTiles = chunkStart[nChunks];
    CASPHY_CUDA_TRY(cudaMemcpyAsync(L.chunkStart, chunkStart.data(), sizeof(u64) * (nChunks + 1),
                                    cudaMemcpyHostToDevice, st));
    k_fill_u64<<<(ntip + 255) / 256, 256, 0, st>>>(L.initKey, ntip, ((u64)ORD_F16_NEG1 << 32) | 0xFFFFFFFFull);
    launches++;
    int initBlocksPerSM = 0;
    CASPHY_CUDA_TRY(cudaEventRecord(ev[1], st));
    InitArgs ia{ntip, ncol, Sp, L.colT0, L.eSC, L.eW, L.eLen, L.chunkStart, nChunks, nTiles, L.tileCounter, L.initKey};
    if (intPath) {
        CASPHY_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&initBlocksPerSM, k_init_scan<true>, kThreads, 0));
        k_init_scan<true><<<nSM * std::max(initBlocksPerSM, 1), kThreads, 0, st>>>(ia);
    } else {
        CASPHY_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&initBlocksPerSM, k_init_scan<false>, kThreads, 0));
        k_init_scan<false><<<nSM * std::max(initBlocksPerSM, 1), kThreads, 0, st>>>(ia);
    }
    launches++;
    CASPHY_CUDA_TRY(cudaEventRecord(ev[2], st));
    const u32 initN = std::max(Sp, nnode);
    k_slot_init<<<(initN + 255) / 256, 256, 0, st>>>(ntip, Sp, nnode, L.initKey, L.lm[0], L.lm[1], L.lm[2],
                                                       L.node2slot, L.nodeDeath, L.nodeSize, L.tipSize);
    launches++;
    JoinArgs ja{};
    ja.ntip = ntip; ja.ncol = ncol; ja.ncolP = ncolP; ja.nState = nState; ja.nnode = nnode; ja.nCTA = nCTA;
    ja.minSize = minSize; ja.minRatio = minRatio; ja.unitW = unitW ? 1 : 0; ja.Wsel = L.Wsel; ja.nodeRow = L.nodeRow;
    ja.colT[0] = L.colT0; ja.colT[1] = L.colT1;
    ja.lmOrd[0] = L.lm[0]; ja.lmIdx[0] = L.lm[1]; ja.slotNode[0] = L.lm[2];
    ja.lmOrd[1] = L.lm[3]; ja.lmIdx[1] = L.lm[4]; ja.slotNode[1] = L.lm[5];
    ja.node2slot = L.node2slot; ja.nodeDeath = L.nodeDeath; ja.nodeSize = L.nodeSize; ja.rawEdge = L.rawEdge;
    ja.pub = L.pub; ja.pubCnt = L.pubCnt; ja.partial = L.partial; ja.counts = L.counts; ja.flags = L.flags;
    ja.err = L.jerr;
    ja.limitNs = 20ull * 1000 * 1000 * 1000;
    ja.statsOut = L.stats; ja.Rmax = Rmax;
    const size_t smemBytes = sizeof(u16) * kCap + sizeof(BlockRec) * 2 * nCTA + sizeof(u32) * ncol +
                             sizeof(u32) * Rmax + sizeof(u16) * (((ncol + 7u) & ~7u) + ncolP) + 2 * nCTA + 64;
    if (ntip >= 2) {
        void* fn = intPath ? (void*)k_join<true> : (void*)k_join<false>;
        CASPHY_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemBytes));
        int perSM = 0;
        CASPHY_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, fn, kThreads, smemBytes));
        if (perSM < 1) {
            casphy_set_last_error_msg("join kernel does not fit on an SM");
            return CASPHY_ERANGE;
        }
        void* args[] = {&ja};
        CASPHY_CUDA_TRY(cudaLaunchCooperativeKernel(fn, dim3(nCTA), dim3(kThreads), args, smemBytes, st));
        launches++;
    }
    CASPHY_CUDA_TRY(cudaEventRecord(ev[3], st));
    std::vector<u32> eLenH(ntip);
    CASPHY_CUDA_TRY(cudaMemcpyAsync(eLenH.data(), L.eLen, sizeof(u32) * ntip, cudaMemcpyDeviceToHost, st));
    std::vector<u32> raw((size_t)2 * nedge + 2);
    unsigned long long hst[8] = {0};
    int herr = 0;
    int hjerr = 0;
    CASPHY_CUDA_TRY(cudaMemcpyAsync(raw.data(), L.rawEdge, sizeof(u32) * 2 * nedge, cudaMemcpyDeviceToHost, st));
    CASPHY_CUDA_TRY(cudaMemcpyAsync(hst, L.stats, sizeof(hst), cudaMemcpyDeviceToHost, st));
    CASPHY_CUDA_TRY(cudaMemcpyAsync(&herr, L.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CASPHY_CUDA_TRY(cudaMemcpyAsync(&hjerr, L.jerr, sizeof(int), cudaMemcpyDeviceToHost, st));
    CASPHY_CUDA_TRY(cudaStreamSynchronize(st));
    if (herr) {
        casphy_set_last_error_msg("cell codes exceed nState+1 (or 65535)");
        return herr;
    }
    if (hjerr) {
        casphy_set_last_error_msg(hjerr == CASPHY_ETIMEOUT ? "join loop grid barrier timed out"
                                                            : "join loop invariant violated");
        return hjerr;
    }
    std::vector<u32> order;
    const u32 nrows = std::max(ntip - 1, 1u);
    if (ntip >= 2) {
        preorder_relabel(ntip, raw.data(), edge_out, order);
        if (order.size() != nrows) return CASPHY_EINTERNAL;
    } else {
        order.assign(1, 0u);
    }
    CASPHY_CUDA_TRY(cudaMemcpyAsync(L.order, order.data(), sizeof(u32) * nrows, cudaMemcpyHostToDevice, st));
    u32* sout = d_state_out ? d_state_out : L.stateOut;
    if (sout) {
        k_gather<<<nrows, 256, 0, st>>>(L.nodeRow, ncol, ncolP, L.order, nrows, sout);
        launches++;
        if (h_state_out)
            CASPHY_CUDA_TRY(cudaMemcpyAsync(h_state_out, sout, sizeof(u32) * (size_t)nrows * ncol,
                                            cudaMemcpyDeviceToHost, st));
    }
    CASPHY_CUDA_TRY(cudaEventRecord(ev[4], st));
    CASPHY_CUDA_TRY(cudaEventSynchronize(ev[4]));
    float t12 = 0, t23 = 0, t04 = 0;
    cudaEventElapsedTime(&t12, ev[1], ev[2]);
    cudaEventElapsedTime(&t23, ev[2], ev[3]);
    cudaEventElapsedTime(&t04, ev[0], ev[4]);
    for (auto& e : ev) cudaEventDestroy(e);
    lst.joins = ntip - 1;
    lst.stale_recomputes = hst[0];
    lst.pair_scores = (u64)ntip * (ntip - 1) / 2 + hst[1];
    lst.compactions = hst[2];
    lst.kernel_launches = launches;
    lst.init_scan_ms = t12;
    lst.join_loop_ms = t23;
    lst.total_ms = t04;
    for (u32 i = 0; i + 1 < ntip; i++) lst.alg_bytes_init += 2ull * eLenH[i] * (u64)(ntip - 1 - i);
    lst.alg_bytes_join = hst[5];
    lst.phases = hst[3];
    lst.refreshes = hst[4];
    if (stats) *stats = lst;
    return CASPHY_OK;
}

}  // namespace casphy

extern "C" int casphy_join_indel(uint32_t ntip, uint32_t ncol, const uint32_t* codes, uint32_t nState,
                                 const double* weight, const uint32_t* tipSize, uint32_t minSize, float minRatio,
                                 uint32_t* edge_out, uint32_t* state_out, casphy_join_stats* stats) {
    int rc = casphy::require_device();
    if (rc) return rc;
    if (!codes || !state_out) return CASPHY_EINVAL;
    casphy::DeviceScope ds;
    return casphy::join_indel_impl(ntip, ncol, nullptr, nState, weight, tipSize, minSize, minRatio, edge_out,
                                   nullptr, state_out, stats, 0, ds, codes);
}

extern "C" int casphy_join_indel_dev(uint32_t ntip, uint32_t ncol, const uint32_t* d_codes, uint32_t nState,
                                     const double* weight, const uint32_t* tipSize, uint32_t minSize,
                                     float minRatio, uint32_t* edge_out, uint32_t* d_state_out,
                                     casphy_join_stats* stats, void* stream) {
    int rc = casphy::require_device();
    if (rc) return rc;
    if (!d_codes) return CASPHY_EINVAL;
    casphy::DeviceScope ds;
    return casphy::join_indel_impl(ntip, ncol, d_codes, nState, weight, tipSize, minSize, minRatio, edge_out,
                                   d_state_out, nullptr, stats, (cudaStream_t)stream, ds, nullptr);
}

// ===========================================================================
// Zero-allocation variant of the indel join.
//
// Some callers cannot allocate device memory while they run us: a framework
// that has already reserved the GPU's memory for its own pool (so a
// cudaMalloc would fail or evict its cache), a latency-critical service loop
// that must not take cudaMalloc/cudaFree's device-wide synchronisation, or
// a host thread that is not allowed to change the device's allocation state.
// For them casphy_join_indel_noalloc runs the same tree build using only the
// buffers the caller passes in plus one fixed scratch region compiled into
// this library.
//
// The scratch region is the file-scope array below.  Every GPU that loads
// libcasphy.so holds it (kScratchBytes) until the process exits.  All calls on
// a device share it and each call overwrites it, so calls whose GPU work
// overlaps (two host threads, or two streams) race; calls are serialised per
// device by a host lock and return only after their work on the stream is
// done.  Every buffer that must start at zero is cleared inside the call.
// ===========================================================================

namespace casphy {
namespace indel_noalloc {

constexpr size_t kScratchBytes = size_t(64) << 20;  // 64 MiB
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Device address of g_scratch for each device, looked up once per device
// (with that device current) on its first call.
static std::mutex g_mu;
static void* g_addr[64] = {nullptr};
static std::mutex g_dev_mu[64];

static int scratch_address(int dev, void** out) {
    std::lock_guard<std::mutex> g(g_mu);
    if (dev < 0 || dev >= 64) return CASPHY_ERANGE;
    if (!g_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) {
            casphy_set_last_cuda_error(e, "cudaGetSymbolAddress(g_scratch)", __FILE__, __LINE__);
            return CASPHY_ECUDA;
        }
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return CASPHY_OK;
}

// binary16 weights, integer weights and the exactness flags, one block per
// site: flags[0] = some weight is not an integer in [0,2048], flags[1] = some
// weight is not 1, flags[2] = some weight is negative or NaN; flags[3] =
// sum over sites of the site's largest weight.
__global__ void k_weights(const double* __restrict__ w, u32 nState, u32 ncol, u16* __restrict__ hbits,
                          u16* __restrict__ wint, u32* flags) {
    const u32 s = blockIdx.x;
    u32 colMax = 0;
    for (u32 a = threadIdx.x; a < nState; a += blockDim.x) {
        const size_t i = (size_t)a * ncol + s;
        const double x = w[i];
        if (!(x >= 0)) atomicOr(flags + 2, 1u);
        const __half h = __double2half(x);
        const float hf = __half2float(h);
        hbits[i] = __half_as_ushort(h);
        const bool isInt = hf == floorf(hf) && hf <= 2048.0f;
        if (!isInt) atomicOr(flags + 0, 1u);
        if (hf != 1.0f) atomicOr(flags + 1, 1u);
        wint[i] = isInt ? (u16)hf : (u16)0;
        colMax = max(colMax, isInt ? (u32)hf : 4096u);
    }
    for (int o = 16; o > 0; o >>= 1) colMax = max(colMax, __shfl_xor_sync(0xFFFFFFFFu, colMax, o));
    if ((threadIdx.x & 31) == 0) atomicAdd(flags + 3, colMax);
}

// Pre-order relabelling on the device (same walk as preorder_relabel).
__global__ void k_preorder(const u32* __restrict__ rawEdge, u32 ntip, u32* relabel, u32* stack,
                           unsigned char* cursor, u32* edge_out, u32* order, u32* err) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const u32 nnode = 2 * ntip - 1;
    for (u32 i = 0; i < nnode; i++) {
        relabel[i] = i < ntip ? i : nnode;
        cursor[i] = 0;
    }
    u32 sp = 0, count = ntip, nout = 0, nord = 0;
    order[nord++] = nnode - 1;
    stack[sp++] = nnode - 1;
    while (sp > 0) {
        const u32 v = stack[sp - 1];
        if (v < ntip || cursor[v] >= 2) { sp--; continue; }
        const u32 ei = 2 * (v - ntip) + cursor[v];
        cursor[v]++;
        const u32 p = rawEdge[2 * ei], c = rawEdge[2 * ei + 1];
        if (p >= nnode || c >= nnode || sp >= nnode) { *err = 1; return; }
        stack[sp++] = c;
        if (relabel[p] == nnode) relabel[p] = count++;
        if (relabel[c] == nnode) {
            order[nord++] = c;
            relabel[c] = count++;
        }
        edge_out[2 * nout] = relabel[p];
        edge_out[2 * nout + 1] = relabel[c];
        nout++;
    }
    if (nout != 2 * ntip - 2 || nord != ntip - 1) *err = 1;
}

struct Layout {
    double* w64; u16* hbits; u16* wint; u32* wflags; u32* tipSize;
    u16* nodeRow; u16* colT0; u16* colT1; u32* lm[6];
    u32* node2slot; u32* nodeDeath; u32* nodeSize; u32* rawEdge;
    u32* eSC; u16* eW; u32* eLen; unsigned long long* initKey;
    BlockRec* pub; u32* pubCnt; u64* partial; u32* counts; u32* flags; int* jerr;
    unsigned long long* tileCounter; u64* chunkStart; unsigned long long* stats;
    u32* relabel; u32* stack; unsigned char* cursor; u32* order; u32* dfsErr; int* prepErr;
    size_t bytes;
};

static Layout carve(char* base, u32 ntip, u32 ncol, u32 nState, u32 nCTA, u32 nChunks) {
    const u32 nnode = 2 * ntip - 1, nedge = 2 * ntip - 2;
    const u32 ncolP = (ncol + 7u) & ~7u, Sp = (ntip + 7u) & ~7u;
    const size_t nw = (size_t)nState * ncol;
    Carve c;
    c.base = base;
    Layout l;
    l.w64 = c.take<double>(nw ? nw : 1);
    l.hbits = c.take<u16>(nw ? nw : 1);
    l.wint = c.take<u16>(nw ? nw : 1);
    l.wflags = c.take<u32>(4);
    l.tipSize = c.take<u32>(ntip);
    l.nodeRow = c.take<u16>((size_t)nnode * ncolP);
    l.colT0 = c.take<u16>((size_t)ncol * Sp);
    l.colT1 = c.take<u16>((size_t)ncol * Sp);
    for (int i = 0; i < 6; i++) l.lm[i] = c.take<u32>(Sp);
    l.node2slot = c.take<u32>(nnode);
    l.nodeDeath = c.take<u32>(nnode);
    l.nodeSize = c.take<u32>(nnode);
    l.rawEdge = c.take<u32>((size_t)2 * nedge + 2);
    l.eSC = c.take<u32>((size_t)ntip * ncol);
    l.eW = c.take<u16>((size_t)ntip * ncol);
    l.eLen = c.take<u32>(ntip);
    l.initKey = c.take<unsigned long long>(ntip);
    l.pub = c.take<BlockRec>(4 * nCTA);
    l.pubCnt = c.take<u32>(2 * nCTA);
    l.partial = c.take<u64>(2 * nCTA);
    l.counts = c.take<u32>(nCTA);
    l.flags = c.take<u32>(16 * nCTA);
    l.jerr = c.take<int>(1);
    l.tileCounter = c.take<unsigned long long>(1);
    l.chunkStart = c.take<u64>(nChunks + 1);
    l.stats = c.take<unsigned long long>(8);
    l.relabel = c.take<u32>(nnode);
    l.stack = c.take<u32>(nnode);
    l.cursor = c.take<unsigned char>(nnode);
    l.order = c.take<u32>(ntip);
    l.dfsErr = c.take<u32>(1);
    l.prepErr = c.take<int>(1);
    l.bytes = c.off + 256;
    return l;
}

}  // namespace indel_noalloc
}  // namespace casphy

extern "C" int casphy_join_indel_noalloc(uint32_t ntip, uint32_t ncol, const uint32_t* d_codes, uint32_t nState,
                                         const double* weight, const uint32_t* tipSize, uint32_t minSize,
                                         float minRatio, uint32_t* d_edge_out, uint32_t* d_state_out,
                                         void* stream) {
    using namespace casphy;
    using namespace casphy::indel;
    using namespace casphy::indel_noalloc;
    if (ntip < 2 || ncol == 0 || !d_codes || !weight || !tipSize || !d_edge_out || !d_state_out)
        return CASPHY_EINVAL;
    if (ncol > kMaxCol) {
        casphy_set_last_error_msg("casphy_join_indel_noalloc: ncol exceeds 16384");
        return CASPHY_ERANGE;
    }
    int dev = 0, nSM = 0;
    CASPHY_CUDA_TRY(cudaGetDevice(&dev));
    CASPHY_CUDA_TRY(cudaDeviceGetAttribute(&nSM, cudaDevAttrMultiProcessorCount, dev));
    const u32 nCTA = (u32)nSM;
    const u32 nChunks = (ntip + kCap - 1) / kCap;
    const Layout need = carve(nullptr, ntip, ncol, nState, nCTA, nChunks);
    if (need.bytes > kScratchBytes) {
        char msg[200];
        snprintf(msg, sizeof(msg),
                 "casphy_join_indel_noalloc: %u cells x %u sites need %zu bytes of scratch, the fixed limit is %zu",
                 ntip, ncol, need.bytes, kScratchBytes);
        casphy_set_last_error_msg(msg);
        return CASPHY_ERANGE;
    }
    void* base = nullptr;
    int rc = scratch_address(dev, &base);
    if (rc) return rc;
    std::lock_guard<std::mutex> devLock(g_dev_mu[dev & 63]);
    cudaStream_t st = (cudaStream_t)stream;
    const Layout L = carve(static_cast<char*>(base), ntip, ncol, nState, nCTA, nChunks);
    const u32 nnode = 2 * ntip - 1;
    const u32 ncolP = (ncol + 7u) & ~7u, Sp = (ntip + 7u) & ~7u;
    const size_t nw = (size_t)nState * ncol;

    // weights: host float64 -> scratch, converted on the device
    if (nw) CASPHY_CUDA_TRY(cudaMemcpyAsync(L.w64, weight, sizeof(double) * nw, cudaMemcpyHostToDevice, st));
    CASPHY_CUDA_TRY(cudaMemcpyAsync(L.tipSize, tipSize, sizeof(u32) * ntip, cudaMemcpyHostToDevice, st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(L.wflags, 0, sizeof(u32) * 4, st));
    if (nw) k_weights<<<ncol, 32, 0, st>>>(L.w64, nState, ncol, L.hbits, L.wint, L.wflags);
    u32 wf[4] = {0, 0, 0, 0};
    CASPHY_CUDA_TRY(cudaMemcpyAsync(wf, L.wflags, sizeof(wf), cudaMemcpyDeviceToHost, st));
    CASPHY_CUDA_TRY(cudaStreamSynchronize(st));
    if (wf[2]) {
        casphy_set_last_error_msg("weights must be >= 0 and not NaN");
        return CASPHY_EINVAL;
    }
    const bool intPath = !wf[0] && wf[3] <= 2048u && (u64)nState + 1 <= 0x7FFFu;
    const bool unitW = intPath && !wf[1];

    // everything the kernels expect to start cleared
    CASPHY_CUDA_TRY(cudaMemsetAsync(L.prepErr, 0, sizeof(int), st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(L.jerr, 0, sizeof(int), st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(L.flags, 0, sizeof(u32) * 16 * nCTA, st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(L.tileCounter, 0, sizeof(unsigned long long), st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(L.stats, 0, sizeof(unsigned long long) * 8, st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(L.dfsErr, 0, sizeof(u32), st));

    PrepArgs pa{ntip, ncol, ncolP, nState, Sp, d_codes, intPath ? L.wint : L.hbits, intPath ? 0x7FFFu : 0xFFFFu,
                L.nodeRow, L.eSC, L.eW, L.eLen, L.prepErr};
    k_prep_rows<<<(ntip + 7) / 8, 256, 0, st>>>(pa);
    k_transpose<<<dim3((Sp + 31) / 32, (ncol + 31) / 32), dim3(32, 8), 0, st>>>(L.nodeRow, ntip, ncol, ncolP, Sp,
                                                                                  L.colT0);
    u64 chunkStart[64 + 1];
    if (nChunks + 1 > 65) return CASPHY_ERANGE;
    chunkStart[0] = 0;
    for (u32 k = 0; k < nChunks; k++) {
        const u64 end = std::min<u64>((u64)(k + 1) * kCap, ntip);
        chunkStart[k + 1] = chunkStart[k] + (end >= 1 ? end - 1 : 0);
    }
    CASPHY_CUDA_TRY(cudaMemcpyAsync(L.chunkStart, chunkStart, sizeof(u64) * (nChunks + 1), cudaMemcpyHostToDevice,
                                    st));
    k_fill_u64<<<(ntip + 255) / 256, 256, 0, st>>>(L.initKey, ntip, ((u64)ORD_F16_NEG1 << 32) | 0xFFFFFFFFull);
    InitArgs ia{ntip, ncol, Sp, L.colT0, L.eSC, L.eW, L.eLen, L.chunkStart, nChunks, chunkStart[nChunks],
                L.tileCounter, L.initKey};
    int perSM = 0;
    if (intPath) {
        CASPHY_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_init_scan<true>, kThreads, 0));
        k_init_scan<true><<<nSM * std::max(perSM, 1), kThreads, 0, st>>>(ia);
    } else {
        CASPHY_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_init_scan<false>, kThreads, 0));
        k_init_scan<false><<<nSM * std::max(perSM, 1), kThreads, 0, st>>>(ia);
    }
    const u32 initN = std::max(Sp, nnode);
    k_slot_init<<<(initN + 255) / 256, 256, 0, st>>>(ntip, Sp, nnode, L.initKey, L.lm[0], L.lm[1], L.lm[2],
                                                       L.node2slot, L.nodeDeath, L.nodeSize, L.tipSize);
    const u32 Rmax = (((ntip + nCTA - 1) / nCTA) + 7u) & ~7u;
    JoinArgs ja{};
    ja.ntip = ntip; ja.ncol = ncol; ja.ncolP = ncolP; ja.nState = nState; ja.nnode = nnode; ja.nCTA = nCTA;
    ja.minSize = minSize; ja.minRatio = minRatio; ja.unitW = unitW ? 1 : 0;
    ja.Wsel = intPath ? L.wint : L.hbits; ja.nodeRow = L.nodeRow;
    ja.colT[0] = L.colT0; ja.colT[1] = L.colT1;
    ja.lmOrd[0] = L.lm[0]; ja.lmIdx[0] = L.lm[1]; ja.slotNode[0] = L.lm[2];
    ja.lmOrd[1] = L.lm[3]; ja.lmIdx[1] = L.lm[4]; ja.slotNode[1] = L.lm[5];
    ja.node2slot = L.node2slot; ja.nodeDeath = L.nodeDeath; ja.nodeSize = L.nodeSize; ja.rawEdge = L.rawEdge;
    ja.pub = L.pub; ja.pubCnt = L.pubCnt; ja.partial = L.partial; ja.counts = L.counts; ja.flags = L.flags;
    ja.err = L.jerr; ja.limitNs = 20ull * 1000 * 1000 * 1000; ja.statsOut = L.stats; ja.Rmax = Rmax;
    const size_t smemBytes = sizeof(u16) * kCap + sizeof(BlockRec) * 2 * nCTA + sizeof(u32) * ncol +
                             sizeof(u32) * Rmax + sizeof(u16) * (((ncol + 7u) & ~7u) + ncolP) + 2 * nCTA + 64;
    void* fn = intPath ? (void*)k_join<true> : (void*)k_join<false>;
    CASPHY_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemBytes));
    void* args[] = {&ja};
    CASPHY_CUDA_TRY(cudaLaunchCooperativeKernel(fn, dim3(nCTA), dim3(kThreads), args, smemBytes, st));
    k_preorder<<<1, 32, 0, st>>>(L.rawEdge, ntip, L.relabel, L.stack, L.cursor, d_edge_out, L.order, L.dfsErr);
    k_gather<<<ntip - 1, 256, 0, st>>>(L.nodeRow, ncol, ncolP, L.order, ntip - 1, d_state_out);
    CASPHY_CUDA_TRY(cudaGetLastError());
    int errs[2] = {0, 0};
    u32 dfsErr = 0;
    CASPHY_CUDA_TRY(cudaMemcpyAsync(&errs[0], L.prepErr, sizeof(int), cudaMemcpyDeviceToHost, st));
    CASPHY_CUDA_TRY(cudaMemcpyAsync(&errs[1], L.jerr, sizeof(int), cudaMemcpyDeviceToHost, st));
    CASPHY_CUDA_TRY(cudaMemcpyAsync(&dfsErr, L.dfsErr, sizeof(u32), cudaMemcpyDeviceToHost, st));
    CASPHY_CUDA_TRY(cudaStreamSynchronize(st));
    if (errs[0]) {
        casphy_set_last_error_msg("cell codes exceed nState+1 (or 65535)");
        return errs[0];
    }
    if (errs[1]) {
        casphy_set_last_error_msg(errs[1] == CASPHY_ETIMEOUT ? "join loop grid barrier timed out"
                                                              : "join loop invariant violated");
        return errs[1];
    }
    return dfsErr ? CASPHY_EINTERNAL : CASPHY_OK;
}
