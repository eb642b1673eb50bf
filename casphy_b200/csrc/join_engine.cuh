// Persistent greedy-join engine shared by the indel and bit joins.
//
// The reference joins (cu/joinEdgeIndel.cu:376-468, cu/joinEdgeBitReverse.cu:
// 404-505) repeat: take the global best local maximum (larger value, then
// smaller node index; reduction seeded with (-1, 0)); if that row's partner
// is already joined, rescore the row against every live row and retry;
// otherwise join the two rows into a new node stored in the first row's
// slot, score the new node against every live row and raise the local maxima
// it strictly improves.
//
// Here one cooperative launch runs the whole loop, one CTA per SM.  CTA b
// owns a contiguous range of slots and everything stored per slot.  Each
// phase ends with an all-to-all flag barrier whose waits are bounded by
// %globaltimer.  After every join each CTA publishes the two best (key,
// slot, partner) records of its range; every CTA keeps an identical table of
// all published records, so it derives the next join by itself.  A stale
// partner costs one scoring phase: the owner stores the row's new maximum and
// every CTA patches its copy of the owner's list (the list keeps its
// invariant "every unlisted live slot ranks below the last entry"; when it
// runs dry the CTAs republish).  When fewer than half the slots are alive
// the slots are renumbered densely (compaction).
//
// A Model supplies the data-specific parts: how a query is built (stale row
// or merged children), where node and slot data live, how one pass of
// candidate scores is computed, and how slot data moves in a compaction.
#pragma once
#include <cstdlib>

#include "common.cuh"

namespace casphy {
namespace joinx {

constexpr int kThreads = 512;
constexpr u32 kDead = 0xFFFFFFFFu;
constexpr u32 kNone = 0xFFFFFFFFu;
constexpr u32 kMaxCap = 4096;  // candidates per scoring pass (ordOut in smem)
constexpr u32 kMaxBatch = 8;   // stale rows rescanned in one phase
constexpr u32 kBatchRecPerLane = 10;  // batch selection reads 2 x nCTA <= 320 table records

// Words of the joined-node bitmap rounded up to keep what follows 16-byte aligned.
__host__ __device__ inline u32 death_words_padded(u32 deathWords) { return (deathWords + 3u) & ~3u; }

struct BlockRec {
    u64 key;
    u32 slot;
    u32 partner;
};

struct Common {
    u32 ntip, nnode, nCTA;
    u32 align;            // slot ranges start at multiples of this (8 or 32)
    u32* lmOrd[2];
    u32* lmIdx[2];
    u32* slotNode[2];
    u32* node2slot;
    u32* nodeDeath;
    u32* nodeSize;
    u32* rawEdge;
    BlockRec* pub;        // 2 phases x nCTA x 2
    u32* pubCnt;          // 2 phases x nCTA
    u64* partial;         // 2 phases x nCTA x kMaxBatch
    u32* counts;          // nCTA
    u32* flags;           // nCTA x 16
    int* err;
    u64 limitNs;
    unsigned long long* statsOut;  // [0] stale [1] pairs [2] compactions [3] phases [4] refreshes [5] alg bytes
    u32 Rmax;
    u32 ordNeg1;          // ordered key of the value -1
    u32 compactMin;       // do not compact below this many slots
    u32 compactQ8;        // compact when alive*256 < slots*compactQ8
    u32 bytesPerPairSite; // algorithmic bytes per (candidate, query entry), x1000
    u32 maxBatch;         // stale rows per rescan phase, 1..kMaxBatch
    u32 deathWords;       // words of the per-CTA shared-memory bitmap of joined nodes (0: none)
    u32 needSizes;        // the model's join reads the two node sizes (minSize > 0)
    u32 keepSizes;        // the caller reads nodeSize of new nodes after the loop (bootstrap clade layout)
    u32 preSlots;         // a join's scan prefetches its slots' node, maximum and partner into shared memory
    unsigned long long* prof;  // nullable: CTA 0 section times (ns), see PROF_*
};

// Sections timed by CTA 0 when Common::prof is set.
enum { PROF_BARRIER = 0, PROF_TABLE, PROF_DECIDE, PROF_BUILD, PROF_SCAN, PROF_POST, PROF_STALE_POST, PROF_COMPACT,
       PROF_SELECT, PROF_STALE_SCAN, PROF_SC_COPY, PROF_SC_ACC, PROF_SC_RED, PROF_N };

// The section sums live in shared memory (only thread 0 of CTA 0 adds to
// them), so the persistent loop does not hold them in registers, and model
// code marks its own sub-sections with prof_mark().
__shared__ unsigned long long prof_acc[PROF_N + 1];  // [PROF_N] = time of the last mark
__shared__ int prof_on;

__device__ __forceinline__ void prof_mark(int sec) {
    if (threadIdx.x != 0 || !prof_on) return;
    const u64 n = globaltimer_ns();
    prof_acc[sec] += n - prof_acc[PROF_N];
    prof_acc[PROF_N] = n;
}

struct Prof {
    bool on;
    __device__ __forceinline__ void init(bool enable) {
        on = enable && threadIdx.x == 0;
        if (threadIdx.x == 0) {
            prof_on = on;
            for (int i = 0; i <= PROF_N; i++) prof_acc[i] = 0;
            if (on) prof_acc[PROF_N] = globaltimer_ns();
        }
        __syncthreads();
    }
    __device__ __forceinline__ void mark(int sec) {
        if (on) prof_mark(sec);
    }
};

struct Range {
    u32 S, Sp, R, lo, hi;
};

__device__ __forceinline__ Range make_range(u32 S, u32 nCTA, u32 b, u32 align) {
    Range r;
    r.S = S;
    r.Sp = (S + align - 1) / align * align;
    const u32 per = (S + nCTA - 1) / nCTA;
    r.R = (per + align - 1) / align * align;
    r.lo = min(b * r.R, S);
    r.hi = min(r.lo + r.R, S);
    return r;
}

__device__ __forceinline__ u32* lmOrd_of(const Common& a, u32 buf) { return buf ? a.lmOrd[1] : a.lmOrd[0]; }
__device__ __forceinline__ u32* lmIdx_of(const Common& a, u32 buf) { return buf ? a.lmIdx[1] : a.lmIdx[0]; }
__device__ __forceinline__ u32* slotNode_of(const Common& a, u32 buf) { return buf ? a.slotNode[1] : a.slotNode[0]; }

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

// Block-wide argmax of records (keys are unique among live slots).
__device__ __forceinline__ BlockRec block_best_rec(u64 best, u32 bslot, u32 bpart, u64* red, BlockRec* s_rec) {
    if (threadIdx.x == 0) { s_rec->slot = kNone; s_rec->partner = 0; }
    const u64 m = block_max_u64(best, red);
    if (best == m && bslot != kNone && m != 0ull) { s_rec->slot = bslot; s_rec->partner = bpart; }
    __syncthreads();
    BlockRec r;
    r.key = m;
    r.slot = s_rec->slot;
    r.partner = s_rec->partner;
    __syncthreads();
    return r;
}

__device__ __forceinline__ void block_top2(Top2 t, u64* red, BlockRec* s_rec, BlockRec* out) {
    const BlockRec r0 = block_best_rec(t.k0, t.s0, t.p0, red, s_rec);
    if (t.k0 == r0.key && t.s0 == r0.slot && r0.key != 0ull) {
        t.k0 = t.k1; t.s0 = t.s1; t.p0 = t.p1;
        t.k1 = 0ull; t.s1 = kNone;
    }
    const BlockRec r1 = block_best_rec(t.k0, t.s0, t.p0, red, s_rec);
    if (threadIdx.x == 0) {
        out[0] = r0;
        out[1] = r1;
    }
    __syncthreads();
}

__device__ __forceinline__ u32 block_sum_u32(u32 v, u32* wsum) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = v;
    __syncthreads();
    u32 t = 0;
    for (int w = 0; w < kThreads / 32; w++) t += wsum[w];
    __syncthreads();
    return t;
}

__device__ __forceinline__ void publish(const Common& a, u32 p, u32 b, const BlockRec* top, u32 cnt) {
    if (threadIdx.x < 2) {
        BlockRec* dst = a.pub + ((size_t)(p & 1) * a.nCTA + b) * 2 + threadIdx.x;
        const BlockRec r = top[threadIdx.x];
        asm volatile("st.global.cg.v2.u64 [%0], {%1, %2};" ::"l"(dst), "l"(r.key),
                     "l"(((u64)r.partner << 32) | r.slot)
                     : "memory");
    }
    if (threadIdx.x == 2) a.pubCnt[(p & 1) * a.nCTA + b] = cnt;
}

struct Table {
    BlockRec* tab;
    unsigned char* cnt;
    unsigned char* exact;
};

__device__ inline void load_table(const Common& a, u32 p, Table t) {
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

// The table of a lone CTA is its own just-published top-2: copied from
// shared memory instead of read back through L2.
__device__ inline void load_table_self(const BlockRec* top, u32 cnt, Table t) {
    if (threadIdx.x < 2) t.tab[threadIdx.x] = top[threadIdx.x];
    if (threadIdx.x == 0) {
        t.cnt[0] = (unsigned char)min(cnt, 2u);
        t.exact[0] = cnt <= 2;
    }
    __syncthreads();
}

__device__ __forceinline__ void load_table_any(const Common& a, u32 p, Table t, const BlockRec* top, u32 cnt) {
    if (a.nCTA == 1) load_table_self(top, cnt, t);
    else load_table(a, p, t);
}

// Top-2 of the stored local maxima of this CTA's slots (refresh/compaction).
__device__ inline void own_top2(const Common& a, u32 buf, const Range& rg, u64* red, BlockRec* s_rec, BlockRec* out,
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
        if (o == a.ordNeg1) continue;
        n++;
        t.push(make_key(o, node), c, ld_cg_u32(li + c));
    }
    *cntOut = block_sum_u32(n, wsum);
    block_top2(t, red, s_rec, out);
}

// The best published record over all blocks; false when some block's best
// is unknown (its list ran dry under stale patches).
__device__ inline bool table_best(const Table& t, u32 nCTA, BlockRec* s_best, u64* red, int* s_flag) {
    if (threadIdx.x == 0) *s_flag = 0;
    __syncthreads();
    u64 best = 0ull;
    u32 bi = kNone;
    for (u32 i = threadIdx.x; i < nCTA; i += kThreads) {
        if (t.cnt[i] == 0) {
            if (!t.exact[i]) *s_flag = 1;
            continue;
        }
        if (t.tab[2 * i].key > best) { best = t.tab[2 * i].key; bi = i; }
    }
    const u64 m = block_max_u64(best, red);
    if (best == m && bi != kNone) *s_best = t.tab[2 * bi];
    __syncthreads();
    return *s_flag == 0 && m != 0ull;
}

// Exclusive ranks of this CTA's live slots (ordered), written to ranks[c-lo]
// (kNone for dead); also moves the per-slot engine arrays to buffer nb.
__device__ inline void compact_slots(const Common& a, u32 buf, u32 nb, const Range& rg, u32 off, u32* ranks, u32* wcount) {
    const u32* sn = slotNode_of(a, buf);
    u32* snN = slotNode_of(a, nb);
    u32* loN = lmOrd_of(a, nb);
    u32* liN = lmIdx_of(a, nb);
    const u32* lo = lmOrd_of(a, buf);
    const u32* li = lmIdx_of(a, buf);
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
        const u32 n = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= (u32)o) incl += n;
    }
    if (lane == 31) wcount[wid] = incl;
    __syncthreads();
    if (threadIdx.x < 32) {
        const u32 wv = threadIdx.x < kThreads / 32 ? wcount[threadIdx.x] : 0u;
        u32 wi = wv;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const u32 n = __shfl_up_sync(0xFFFFFFFFu, wi, o);
            if (lane >= (u32)o) wi += n;
        }
        if (threadIdx.x < kThreads / 32) wcount[16 + threadIdx.x] = wi - wv;
    }
    __syncthreads();
    u32 r = off + wcount[16 + wid] + incl - v;
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
}

// The rows rescanned in a stale phase: every visible record (the table holds
// each CTA's top two) whose partner has joined and whose key beats the best
// visible fresh record, best first, at most maxB.  out[0] is the table's best
// record.  Rescanning a stale row before the sequential loop would reach it
// gives the same record the later rescan would (the value is the best over
// the live rows, ties go to the smaller node and new nodes only replace a
// record by a strictly larger value), and a join is taken only when the best
// record is fresh, so the joins come in the sequential order.  Warp 0 selects;
// every CTA reads the same table and so selects the same rows.
__device__ inline u32 stale_batch(const Common& a, const Table& t, const u32* deathBits, u32 k, u32 S, u32 maxB,
                                  BlockRec* out, u32* s_n) {
    if (threadIdx.x < 32) {
        const u32 lane = threadIdx.x, nrec = 2 * a.nCTA;
        u64 fresh = 0ull;
        // every partner's death and slot loaded before any is used
        u32 pn[kBatchRecPerLane], dv[kBatchRecPerLane], sv[kBatchRecPerLane];
        bool ok[kBatchRecPerLane];
#pragma unroll
        for (u32 j = 0; j < kBatchRecPerLane; j++) {
            const u32 i = lane + 32 * j;
            ok[j] = i < nrec && (i & 1u) < t.cnt[i >> 1];
            pn[j] = ok[j] ? t.tab[i].partner : 0u;
        }
        if (a.deathWords) {
            // joined nodes from this CTA's own bitmap: no L2 round trip
#pragma unroll
            for (u32 j = 0; j < kBatchRecPerLane; j++) {
                dv[j] = ok[j] && ((deathBits[pn[j] >> 5] >> (pn[j] & 31)) & 1u) ? 0u : kNone;
                sv[j] = 0u;
            }
        } else {
#pragma unroll
            for (u32 j = 0; j < kBatchRecPerLane; j++) {
                dv[j] = ok[j] ? ld_cg_u32(a.nodeDeath + pn[j]) : 0u;
                sv[j] = ok[j] ? ld_cg_u32(a.node2slot + pn[j]) : 0u;
            }
        }
        // candidate keys (stale, above the best fresh record) stay in registers
        u64 ck[kBatchRecPerLane];
#pragma unroll
        for (u32 j = 0; j < kBatchRecPerLane; j++) {
            const u64 key = ok[j] ? t.tab[lane + 32 * j].key : 0ull;
            const bool st = ok[j] && (dv[j] < k || sv[j] >= S);
            ck[j] = st ? key : 0ull;
            if (ok[j] && !st) fresh = key > fresh ? key : fresh;
        }
        fresh = warp_max_u64(fresh);
#pragma unroll
        for (u32 j = 0; j < kBatchRecPerLane; j++) ck[j] = ck[j] > fresh ? ck[j] : 0ull;
        u32 n = 0;
        while (n < maxB) {
            u64 best = 0ull;
#pragma unroll
            for (u32 j = 0; j < kBatchRecPerLane; j++) best = ck[j] > best ? ck[j] : best;
            const u64 top = warp_max_u64(best);
            if (top == 0ull) break;
            // keys of live rows are unique: exactly one lane holds it
#pragma unroll
            for (u32 j = 0; j < kBatchRecPerLane; j++) {
                if (ck[j] == top) {
                    out[n] = t.tab[lane + 32 * j];
                    ck[j] = 0ull;
                }
            }
            n++;
        }
        if (lane == 0) *s_n = n;
    }
    __syncthreads();
    const u32 n = *s_n;
    __syncthreads();
    return n;
}

// Rescans of nb stale rows one query at a time (models without a fused
// multi-query scan): best[q] gets the top (score, node) key over this CTA's
// live slots other than row q's own.
template <class M>
__device__ inline void stale_scan_each(const Common& a, const typename M::Args& m, typename M::Smem& ms, u32 buf,
                                       const Range& rg, u32 nb, const BlockRec* rows, u64* best, int* nEout,
                                       u32* ordOut, u64* red, BlockRec* s_rec, u32* wcount) {
    const u32* sn = slotNode_of(a, buf);
    for (u32 q = 0; q < nb; q++) {
        const u32 c1 = rows[q].slot;
        const int nE = M::build_stale(m, ms, key_node(rows[q].key), wcount);
        Top2 tt;
        tt.init();
        const u32 cap = M::pass_cap(m, rg.hi - rg.lo);
        for (u32 base = rg.lo; base < rg.hi; base += cap) {
            M::score_pass(m, ms, buf, rg, base, cap, nE, ordOut);
            for (u32 x = threadIdx.x; x < cap && base + x < rg.hi; x += kThreads) {
                const u32 c = base + x;
                const u32 node = ld_cg_u32(sn + c);
                if (node == kDead || c == c1) continue;
                tt.push(make_key(ordOut[x], node), c, 0u);
            }
            __syncthreads();
        }
        const BlockRec pr = block_best_rec(tt.k0, tt.s0, 0u, red, s_rec);
        if (threadIdx.x == 0) {
            best[q] = pr.key;
            nEout[q] = nE;
        }
    }
    __syncthreads();
}

// The join loop for CTA b of a.nCTA co-resident CTAs (b = 0 of 1 when one
// CTA runs a whole join by itself).  smem: engine + model dynamic memory.
template <class M>
__device__ __forceinline__ void join_run(const Common& a, const typename M::Args& m, u32 b, unsigned char* smem) {
    u32* ordOut = reinterpret_cast<u32*>(smem);                        // kMaxCap
    u32* deathBits = ordOut + kMaxCap;                                 // joined nodes (deathWords)
    u32* preSn = deathBits + death_words_padded(a.deathWords);         // 3 x Rmax when a.preSlots
    u32* preLo = preSn + a.Rmax;
    u32* preLi = preLo + a.Rmax;
    BlockRec* tabRec = reinterpret_cast<BlockRec*>(preSn + (a.preSlots ? 3 * a.Rmax : 0u));  // 2*nCTA
    u32* ranks = reinterpret_cast<u32*>(tabRec + 2 * a.nCTA);          // Rmax
    unsigned char* tabCnt = reinterpret_cast<unsigned char*>(ranks + a.Rmax);
    unsigned char* tabExact = tabCnt + a.nCTA;
    unsigned char* msm = smem + M::engine_smem_bytes(a.nCTA, a.Rmax, a.deathWords, a.preSlots);  // model part
    typename M::Smem ms;
    M::carve_smem(m, msm, ms);
    __shared__ u64 red[32];
    __shared__ BlockRec s_rec, s_best;
    __shared__ BlockRec s_top[2];
    __shared__ u32 wcount[40];
    __shared__ u32 wsum[16];
    __shared__ u32 s_val[4];
    __shared__ int s_flag;
    __shared__ BlockRec s_batch[kMaxBatch];
    __shared__ u64 s_pbest[kMaxBatch];
    __shared__ int s_nE[kMaxBatch];
    __shared__ u32 s_nb;

    const Table T{tabRec, tabCnt, tabExact};
    const u32 nCTA = a.nCTA;
    Prof pf;
    pf.init(a.prof != nullptr && b == 0);
    u32 buf = 0;
    Range rg = make_range(a.ntip, nCTA, b, a.align);
    u32 k = 0, p = 0;
    unsigned long long nStale = 0, nPairs = 0, nComp = 0, nRefresh = 0, algMilli = 0;
    const u32 nJoin = a.ntip - 1;
    int fail = 0;
    u32 cnt = 0;

    for (u32 i = threadIdx.x; i < a.deathWords; i += kThreads) deathBits[i] = 0u;
    own_top2(a, buf, rg, red, &s_rec, s_top, &cnt, wsum);
    publish(a, p, b, s_top, cnt);
    if (flag_barrier(a.flags, nCTA, b, ++p, a.err, a.limitNs)) goto out;
    load_table_any(a, p - 1, T, s_top, cnt);

    pf.mark(PROF_COMPACT);
    while (k < nJoin) {
        const bool known = table_best(T, nCTA, &s_best, red, &s_flag);
        pf.mark(PROF_DECIDE);
        if (!known) {
            own_top2(a, buf, rg, red, &s_rec, s_top, &cnt, wsum);
            publish(a, p, b, s_top, cnt);
            nRefresh++;
            pf.mark(PROF_POST);
            if (flag_barrier(a.flags, nCTA, b, ++p, a.err, a.limitNs)) goto out;
            pf.mark(PROF_BARRIER);
            load_table_any(a, p - 1, T, s_top, cnt);
            pf.mark(PROF_TABLE);
            continue;
        }
        const BlockRec g = s_best;
        const u32 j1 = key_node(g.key), c1 = g.slot, j2 = g.partner;
        if (c1 >= rg.S || j1 >= a.nnode || j2 >= a.nnode) { fail = CASPHY_EINTERNAL; break; }
        // With the joined-node bitmap and no size rule, the decision needs no
        // load: the partner's slot (and, for callers that read the new node's
        // size, the two node sizes) is loaded by thread 0 and first used after
        // the query build, which hides its latency.
        const bool quick = a.deathWords && !a.needSizes;
        bool stale;
        u32 c2 = 0, s1 = 0, s2 = 0, c2pending = 0, s1pending = 0, s2pending = 0;
        if (quick) {
            stale = (deathBits[j2 >> 5] >> (j2 & 31)) & 1u;
            if (!stale && threadIdx.x == 0) {
                c2pending = ld_cg_u32(a.node2slot + j2);
                if (a.keepSizes) {
                    s1pending = ld_cg_u32(a.nodeSize + j1);
                    s2pending = ld_cg_u32(a.nodeSize + j2);
                }
            }
        } else {
            if (threadIdx.x == 0) {
                s_val[0] = ld_cg_u32(a.nodeDeath + j2);
                s_val[1] = ld_cg_u32(a.node2slot + j2);
                s_val[2] = ld_cg_u32(a.nodeSize + j1);
                s_val[3] = ld_cg_u32(a.nodeSize + j2);
            }
            __syncthreads();
            const u32 death = s_val[0];
            c2 = s_val[1]; s1 = s_val[2]; s2 = s_val[3];
            __syncthreads();
            stale = death < k || c2 >= rg.S;
        }
        pf.mark(PROF_DECIDE);
        if (stale) {
            // rescan a batch of stale rows (the best record first) against every live slot
            u32 nb = 1;
            if (a.maxBatch > 1 && 2 * nCTA <= 32 * kBatchRecPerLane) {
                nb = stale_batch(a, T, deathBits, k, rg.S, a.maxBatch, s_batch, &s_nb);
            } else {
                if (threadIdx.x == 0) s_batch[0] = g;
                __syncthreads();
            }
            if (nb == 0 || s_batch[0].slot != c1) { fail = CASPHY_EINTERNAL; break; }
            pf.mark(PROF_SELECT);
            if constexpr (M::kFusedStale) {
                if (nb >= 1)
                    M::stale_multi(m, ms, buf, rg, slotNode_of(a, buf), nb, s_batch, s_pbest, s_nE, ordOut, red,
                                   wcount);
                else
                    stale_scan_each<M>(a, m, ms, buf, rg, 1, s_batch, s_pbest, s_nE, ordOut, red, &s_rec, wcount);
            } else {
                stale_scan_each<M>(a, m, ms, buf, rg, nb, s_batch, s_pbest, s_nE, ordOut, red, &s_rec, wcount);
            }
            pf.mark(PROF_STALE_SCAN);
            if (threadIdx.x < nb) {
                asm volatile("st.global.cg.u64 [%0], %1;" ::"l"(a.partial + ((p & 1) * nCTA + b) * kMaxBatch +
                                                                  threadIdx.x),
                             "l"(s_pbest[threadIdx.x])
                             : "memory");
            }
            for (u32 q = 0; q < nb; q++) {
                nStale++;
                nPairs += (a.ntip - k) - 1;
                algMilli += (unsigned long long)a.bytesPerPairSite * (u64)s_nE[q] * ((a.ntip - k) - 1);
            }
            if (flag_barrier(a.flags, nCTA, b, ++p, a.err, a.limitNs)) goto out;
            pf.mark(PROF_BARRIER);
            // warp q reduces row q's partial bests over the CTAs
            {
                const u32 wq = threadIdx.x >> 5, lane = threadIdx.x & 31;
                if (wq < nb) {
                    u64 pb = make_key(a.ordNeg1, 0u);
                    if (nCTA == 1) {
                        pb = s_pbest[wq] > pb ? s_pbest[wq] : pb;  // the lone CTA's own best
                    } else {
                        // all of a lane's loads issued before any is used
                        const u64* src = a.partial + ((p - 1) & 1) * nCTA * kMaxBatch + wq;
                        u64 v[kBatchRecPerLane / 2];
#pragma unroll
                        for (u32 j = 0; j < kBatchRecPerLane / 2; j++) {
                            const u32 i = lane + 32 * j;
                            v[j] = i < nCTA ? ld_cg_u64(src + (size_t)i * kMaxBatch) : 0ull;
                        }
#pragma unroll
                        for (u32 j = 0; j < kBatchRecPerLane / 2; j++) pb = v[j] > pb ? v[j] : pb;
                        for (u32 i = lane + 16 * kBatchRecPerLane; i < nCTA; i += 32) {
                            const u64 x = ld_cg_u64(src + (size_t)i * kMaxBatch);
                            pb = x > pb ? x : pb;
                        }
                        pb = warp_max_u64(pb);
                    }
                    __syncwarp();
                    if (lane == 0) s_pbest[wq] = pb;
                }
            }
            __syncthreads();
            // owners store the new maxima; every CTA patches its table copy in batch order
            if (threadIdx.x < nb) {
                const BlockRec row = s_batch[threadIdx.x];
                if (row.slot / rg.R == b) {
                    lmOrd_of(a, buf)[row.slot] = key_ord(s_pbest[threadIdx.x]);
                    lmIdx_of(a, buf)[row.slot] = key_node(s_pbest[threadIdx.x]);
                }
            }
            if (threadIdx.x == 0) {
                for (u32 q = 0; q < nb; q++) {
                    const BlockRec row = s_batch[q];
                    const u32 vOrd = key_ord(s_pbest[q]), vIdx = key_node(s_pbest[q]);
                    const u32 ob = row.slot / rg.R;
                    BlockRec nr;
                    nr.key = make_key(vOrd, key_node(row.key));
                    nr.slot = row.slot;
                    nr.partner = vIdx;
                    BlockRec* L = T.tab + 2 * ob;
                    unsigned char n = T.cnt[ob];
                    // drop the row's old record (it is listed: it was selected from this table)
                    if (n >= 1 && L[0].slot == row.slot) {
                        L[0] = L[1];
                        n--;
                    } else if (n == 2 && L[1].slot == row.slot) {
                        n--;
                    } else {
                        fail = CASPHY_EINTERNAL;
                    }
                    const bool real = vOrd != a.ordNeg1;
                    if (T.exact[ob]) {
                        if (real) {
                            if (n == 0) L[0] = nr;
                            else if (nr.key > L[0].key) { L[1] = L[0]; L[0] = nr; }
                            else L[1] = nr;
                            n++;
                        }
                    } else if (n >= 1 && real && nr.key > L[n - 1].key) {
                        // above the last listed record, hence above every unlisted one
                        if (nr.key > L[0].key) { L[1] = L[0]; L[0] = nr; }
                        else L[1] = nr;
                        n = 2;
                    }
                    T.cnt[ob] = n;
                }
            }
            if (__syncthreads_or(fail)) break;
            pf.mark(PROF_STALE_POST);
            continue;
        }
        // join j1 and j2 into node ntip+k
        const u32 newNode = a.ntip + k;
        const int nE = M::build_join(m, ms, j1, j2, s1, s2, wcount);
        if (quick) {
            if (threadIdx.x == 0) {
                s_val[1] = c2pending;
                s_val[2] = s1pending;
                s_val[3] = s2pending;
            }
            __syncthreads();
            c2 = s_val[1];
            s1 = s_val[2];
            s2 = s_val[3];
            if (c2 >= rg.S) fail = CASPHY_EINTERNAL;  // a live node always has a slot
            __syncthreads();
            if (fail) break;
        }
        pf.mark(PROF_BUILD);
        // CTA 0 writes the new node's row and the owner of c1 its slot data
        // (slicing them over every CTA was measured slower)
        if (b == 0) {
            M::store_node(m, ms, newNode, 0, 1);
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
            M::store_slot(m, ms, buf, rg, c1, 0, 1);
            if (threadIdx.x == 0) {
                slotNode_of(a, buf)[c1] = newNode;
                lmOrd_of(a, buf)[c1] = a.ordNeg1;
            }
        }
        if (c2 >= rg.lo && c2 < rg.hi && threadIdx.x == 0) {
            slotNode_of(a, buf)[c2] = kDead;
            lmOrd_of(a, buf)[c2] = a.ordNeg1;
        }
        __syncthreads();
        {
            Top2 tt;
            tt.init();
            u32 n = 0;
            const u32* sn = slotNode_of(a, buf);
            u32* lop = lmOrd_of(a, buf);
            u32* lip = lmIdx_of(a, buf);
            const u32 cap = M::pass_cap(m, rg.hi - rg.lo);
            // one pass over the range: its slots' node, maximum and partner are
            // copied into shared memory in the scan's first load round (the
            // model waits for every copy of this thread before it returns)
            const bool pre = a.preSlots && cap >= rg.hi - rg.lo;
            if (pre && rg.lo < rg.hi) {
                const u32 n4 = (rg.hi - rg.lo + 3u) / 4u;
                for (u32 i = threadIdx.x; i < 3 * n4; i += kThreads) {
                    const u32 arr = i / n4, j = 4 * (i % n4);
                    const u32* src = arr == 0 ? sn : (arr == 1 ? lop : lip);
                    cp_async16(preSn + arr * a.Rmax + j, src + rg.lo + j);
                }
            }
            for (u32 base = rg.lo; base < rg.hi; base += cap) {
                M::score_pass(m, ms, buf, rg, base, cap, nE, ordOut);
                for (u32 x = threadIdx.x; x < cap && base + x < rg.hi; x += kThreads) {
                    const u32 c = base + x;
                    const u32 node = pre ? preSn[x] : ld_cg_u32(sn + c);
                    u32 lo = pre ? preLo[x] : ld_cg_u32(lop + c);
                    u32 li = pre ? preLi[x] : ld_cg_u32(lip + c);
                    // c1 and c2 changed this phase (the copies may predate the changes)
                    if (node == kDead || c == c1 || c == c2) continue;
                    const u32 o = ordOut[x];
                    if (o > lo) {  // strict improvement
                        lo = o;
                        li = newNode;
                        lop[c] = o;
                        lip[c] = newNode;
                    }
                    if (lo != a.ordNeg1) {
                        n++;
                        tt.push(make_key(lo, node), c, li);
                    }
                }
                __syncthreads();
            }
            pf.mark(PROF_SCAN);
            cnt = block_sum_u32(n, wsum);
            block_top2(tt, red, &s_rec, s_top);
        }
        publish(a, p, b, s_top, cnt);
        pf.mark(PROF_POST);
        nPairs += (a.ntip - k - 1) - 1;
        algMilli += (unsigned long long)a.bytesPerPairSite * (u64)nE * ((a.ntip - k - 1) - 1);
        if (a.deathWords && threadIdx.x == 0) {
            deathBits[j1 >> 5] |= 1u << (j1 & 31);
            deathBits[j2 >> 5] |= 1u << (j2 & 31);
        }
        k++;
        if (flag_barrier(a.flags, nCTA, b, ++p, a.err, a.limitNs)) goto out;
        pf.mark(PROF_BARRIER);
        load_table_any(a, p - 1, T, s_top, cnt);
        pf.mark(PROF_TABLE);

        // renumber slots densely when too few are alive
        const u32 alive = a.ntip - k;
        if (k < nJoin && rg.S >= a.compactMin && (u64)alive * 256 < (u64)rg.S * a.compactQ8) {
            {
                const u32* sn = slotNode_of(a, buf);
                u32 v = 0;
                for (u32 c = rg.lo + threadIdx.x; c < rg.hi; c += kThreads) v += ld_cg_u32(sn + c) != kDead;
                v = block_sum_u32(v, wsum);
                if (threadIdx.x == 0) a.counts[b] = v;
                M::compact_prepare(m, ms, buf ^ 1u, make_range(alive, nCTA, b, a.align));
            }
            if (flag_barrier(a.flags, nCTA, b, ++p, a.err, a.limitNs)) goto out;
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
            const u32 nb = buf ^ 1u;
            const Range nr = make_range(Snew, nCTA, b, a.align);
            compact_slots(a, buf, nb, rg, off, ranks, wcount);
            M::compact_move(m, ms, buf, nb, rg, nr.Sp, ranks, slotNode_of(a, buf));
            if (b == 0) {
                for (u32 x = Snew + threadIdx.x; x < nr.Sp; x += kThreads) {
                    slotNode_of(a, nb)[x] = kDead;
                    lmOrd_of(a, nb)[x] = a.ordNeg1;
                }
            }
            if (flag_barrier(a.flags, nCTA, b, ++p, a.err, a.limitNs)) goto out;
            buf = nb;
            rg = make_range(Snew, nCTA, b, a.align);
            M::after_compact(m, ms, buf, rg);
            own_top2(a, buf, rg, red, &s_rec, s_top, &cnt, wsum);
            publish(a, p, b, s_top, cnt);
            nComp++;
            if (flag_barrier(a.flags, nCTA, b, ++p, a.err, a.limitNs)) goto out;
            load_table_any(a, p - 1, T, s_top, cnt);
            pf.mark(PROF_COMPACT);
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
        a.statsOut[5] = algMilli / 1000ull;
    }
    if (pf.on)
        for (int i = 0; i < PROF_N; i++) a.prof[i] = prof_acc[i];
}

template <class M>
__global__ void __launch_bounds__(kThreads, 1) k_join(Common a, typename M::Args m) {
    extern __shared__ __align__(16) unsigned char smem[];
    join_run<M>(a, m, blockIdx.x, smem);
}

// Host: stale rows per rescan phase (CASPHY_STALE_BATCH, 1..kMaxBatch;
// default kMaxBatch).
inline u32 stale_batch_setting() {
    const char* e = getenv("CASPHY_STALE_BATCH");
    if (!e) return kMaxBatch;
    const long v = strtol(e, nullptr, 10);
    return v < 1 ? 1u : (v > (long)kMaxBatch ? kMaxBatch : (u32)v);
}

// Host: bytes of engine shared memory before the model's part.
__host__ __device__ inline size_t engine_smem(u32 nCTA, u32 Rmax, u32 deathWords = 0, u32 preSlots = 0) {
    size_t s = sizeof(u32) * kMaxCap + sizeof(u32) * death_words_padded(deathWords) +
               (preSlots ? sizeof(u32) * 3 * (size_t)Rmax : 0) + sizeof(BlockRec) * 2 * nCTA + sizeof(u32) * Rmax +
               2 * nCTA;
    return (s + 15) & ~size_t(15);
}

__global__ void k_slot_init(u32 ntip, u32 Sp, u32 nnode, const unsigned long long* initKey, u32 ordNeg1, u32* lmOrd,
                            u32* lmIdx, u32* slotNode, u32* node2slot, u32* nodeDeath, u32* nodeSize,
                            const u32* tipSize);
__global__ void k_fill_u64(unsigned long long* p, u64 n, u64 v);

// Pre-order walk of the raw join edges (cu/joinEdgeIndel.cu:488-558).
void preorder_relabel(u32 ntip, const u32* rawEdge, u32* edge_out, u32* order);

}  // namespace joinx
}  // namespace casphy
