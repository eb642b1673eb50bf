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
//  * The join loop (cu/joinEdgeIndel.cu:376-468) runs in the persistent join
//    engine (join_engine.cuh) with the IndelDense model below: every CTA
//    merges the two children itself, builds the query site list in shared
//    memory and scores its own slots.  Dead slots are squeezed out of the
//    column matrix whenever fewer than 3/4 of the slots are alive.
//  * Pre-order relabelling (cu/joinEdgeIndel.cu:488-558) walks the 2(N-1)
//    raw edges on the host in O(N) and gathers the state rows on device.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "join_engine.cuh"
#include "runtime.h"

namespace casphy {
namespace indel {

constexpr int kThreads = 512;
constexpr int kG = 8;                       // candidates per thread (one uint4 of u16)
constexpr int kCap = kThreads * kG;         // candidates per pass
constexpr u32 kNone = 0xFFFFFFFFu;
constexpr u32 kMaxCol = 16384;

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
// persistent join loop: the dense (column-major u16) model for the engine

__device__ __forceinline__ u32 merge_code(int mode, u32 x, u32 y) {
    if (mode == 0 || mode == 2) return x;
    if (mode == 1) return y;
    return (x == 0) ? y : ((y >= 1 && x != y) ? 1u : x);
}

// Builds the query site list (ascending sites with code > 1) from a row.
// mode 0: query = row1; 1: copy row2; 2: keep row1; 3: ancestral merge of
// row1 and row2 (updateAncestralKernel, cu/joinEdgeIndel.cu:87-99).  When
// mrow is given the row is also left there for the write-back, and when orow
// is given row1 itself (all ncolP entries) is left there too.
// With at most kPerSmall sites per thread (ncolP <= 2048) every thread issues
// all its row loads before it uses one, so the build costs one L2 round trip.
constexpr u32 kPerSmall = 4;
__device__ int build_indel_query(u32 ncol, u32 ncolP, int unitW, const u16* Wsel, const u16* row1, const u16* row2,
                                 int mode, u16* mrow, u16* orow, u32* eSC, u16* eW, u32* wcount) {
    const u32 lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const u32 per = (ncolP + kThreads - 1) / kThreads;
    const u32 s0 = threadIdx.x * per;
    const bool wantX = mode != 1 || orow != nullptr, wantY = mode == 1 || mode == 3;
    u32 cnt = 0;
    u32 codes[kPerSmall];
    const bool small = per <= kPerSmall;
    if (small) {
        u32 xs[kPerSmall], ys[kPerSmall];
#pragma unroll
        for (u32 i = 0; i < kPerSmall; i++) {
            const u32 s = s0 + i;
            xs[i] = (i < per && s < ncolP && wantX) ? (u32)ld_cg_u16(row1 + s) : 0u;
            ys[i] = (i < per && s < ncol && wantY) ? (u32)ld_cg_u16(row2 + s) : 0u;
        }
#pragma unroll
        for (u32 i = 0; i < kPerSmall; i++) {
            const u32 s = s0 + i;
            const u32 c = (i < per && s < ncol) ? merge_code(mode, xs[i], ys[i]) : 0u;
            if (i < per && s < ncolP) {
                if (mrow) mrow[s] = (u16)c;
                if (orow) orow[s] = (u16)xs[i];
            }
            codes[i] = c;
            cnt += c > 1;
        }
    } else {
        for (u32 i = 0; i < per; i++) {
            const u32 s = s0 + i;
            const u32 x = (s < ncolP && wantX) ? (u32)ld_cg_u16(row1 + s) : 0u;
            const u32 y = (s < ncol && wantY) ? (u32)ld_cg_u16(row2 + s) : 0u;
            const u32 c = s < ncol ? merge_code(mode, x, y) : 0u;
            if (s < ncolP) {
                if (mrow) mrow[s] = (u16)c;
                if (orow) orow[s] = (u16)x;
            }
            cnt += c > 1;
        }
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
    if (small) {
#pragma unroll
        for (u32 i = 0; i < kPerSmall; i++) {
            const u32 s = s0 + i, c = codes[i];
            if (c > 1) {
                eSC[pos] = s | (c << 16);
                eW[pos] = unitW ? (u16)1 : Wsel[(size_t)(c - 2) * ncol + s];
                pos++;
            }
        }
    } else {
        for (u32 i = 0; i < per; i++) {
            const u32 s = s0 + i;
            const u32 c = (s < ncolP && mrow) ? mrow[s] : (s < ncol ? ld_cg_u16(row1 + s) : 0u);
            if (c > 1) {
                eSC[pos] = s | (c << 16);
                eW[pos] = unitW ? (u16)1 : Wsel[(size_t)(c - 2) * ncol + s];
                pos++;
            }
        }
    }
    const int n = (int)wcount[32];
    __syncthreads();
    return n;
}

template <bool INTP>
struct IndelDense {
    static constexpr bool kFusedStale = false;  // stale batches rescan one query at a time
    struct Args {
        u32 ncol, ncolP, nState, minSize;
        float minRatio;
        int unitW;
        const u16* Wsel;
        u16* nodeRow;
        u16* colT[2];
    };
    struct Smem {
        u16* part;
        u32* eSC;
        u16* eW;
        u16* mrow;
    };
    __host__ __device__ static size_t engine_smem_bytes(u32 nCTA, u32 Rmax, u32 deathWords = 0, u32 pre = 0) {
        return joinx::engine_smem(nCTA, Rmax, deathWords, pre);
    }
    __host__ static size_t model_smem_bytes(const Args& m) {
        return sizeof(u16) * kCap + sizeof(u32) * m.ncol + sizeof(u16) * (((m.ncol + 7u) & ~7u) + m.ncolP) + 16;
    }
    __device__ static void carve_smem(const Args& m, unsigned char* p, Smem& s) {
        s.part = reinterpret_cast<u16*>(p);
        s.eSC = reinterpret_cast<u32*>(s.part + kCap);
        s.eW = reinterpret_cast<u16*>(s.eSC + m.ncol);
        s.mrow = s.eW + ((m.ncol + 7u) & ~7u);
    }
    __device__ static u16* col(const Args& m, u32 buf) { return buf ? m.colT[1] : m.colT[0]; }
    __device__ static int build_stale(const Args& m, Smem& s, u32 j1, u32* wc) {
        return build_indel_query(m.ncol, m.ncolP, m.unitW, m.Wsel, m.nodeRow + (size_t)j1 * m.ncolP, nullptr, 0,
                                 nullptr, nullptr, s.eSC, s.eW, wc);
    }
    // minSize / minRatio rule of cu/joinEdgeIndel.cu:407-413
    __device__ static int build_join(const Args& m, Smem& s, u32 j1, u32 j2, u32 s1, u32 s2, u32* wc) {
        int mode;
        if (s1 < m.minSize && __uint2float_rn(s1) * m.minRatio < __uint2float_rn(s2)) mode = 1;
        else if (s2 < m.minSize && __uint2float_rn(s2) * m.minRatio < __uint2float_rn(s1)) mode = 2;
        else mode = 3;
        return build_indel_query(m.ncol, m.ncolP, m.unitW, m.Wsel, m.nodeRow + (size_t)j1 * m.ncolP,
                                 m.nodeRow + (size_t)j2 * m.ncolP, mode, s.mrow, nullptr, s.eSC, s.eW, wc);
    }
    // slice `part` of `nparts` of the new node's row (the engine writes it whole)
    __device__ static void store_node(const Args& m, Smem& s, u32 newNode, u32 part, u32 nparts) {
        u16* dst = m.nodeRow + (size_t)newNode * m.ncolP;
        const u32 per = (m.ncolP + nparts - 1) / nparts, i1 = min(m.ncolP, (part + 1) * per);
        for (u32 i = part * per + threadIdx.x; i < i1; i += kThreads) dst[i] = s.mrow[i];
    }
    // slice `part` of `nparts` of slot c1's column entries (the engine gives
    // the whole column to c1's owner)
    __device__ static void store_slot(const Args& m, Smem& s, u32 buf, const joinx::Range& rg, u32 c1, u32 part,
                                      u32 nparts) {
        u16* c = col(m, buf);
        const u32 per = (m.ncol + nparts - 1) / nparts, i1 = min(m.ncol, (part + 1) * per);
        for (u32 i = part * per + threadIdx.x; i < i1; i += kThreads) c[(size_t)i * rg.Sp + c1] = s.mrow[i];
    }
    // INT: the query entries are split over F thread groups that share the
    // candidates (F as large as the CTA's slot range allows); HALF: one group,
    // because binary16 sums must be formed in ascending site order.
    __host__ __device__ static u32 pass_cap(const Args&, u32 R) {
        u32 F = 1;
        if (INTP) {
            while (F < 16 && (u32)(kCap / (F * 2)) >= R) F *= 2;
        }
        return kCap / F;
    }
    __device__ static void score_pass(const Args& m, Smem& s, u32 buf, const joinx::Range& rg, u32 base, u32 cap,
                                      int nE, u32* ordOut) {
        const u32 F = kCap / cap, Tg = kThreads / F;
        const u32 g = threadIdx.x / Tg, t = threadIdx.x % Tg;
        const u32 cb = base + t * kG;
        Acc8<INTP> acc;
        acc.zero();
        if (cb < rg.hi) accumulate<INTP>(acc, col(m, buf), rg.Sp, cb, s.eSC, s.eW, (int)g, nE, (int)F);
        acc.store(s.part + g * cap + t * kG);
        __syncthreads();
        for (u32 x = threadIdx.x; x < cap && base + x < rg.hi; x += kThreads) {
            u32 hb;
            if (INTP) {
                u32 sum = 0;
                for (u32 gg = 0; gg < F; gg++) sum += s.part[gg * cap + x];
                hb = half_bits_of_int(sum);
            } else {
                hb = s.part[x];
            }
            ordOut[x] = ord_f16((u16)hb);
        }
        __syncthreads();
    }
    __device__ static void compact_prepare(const Args&, Smem&, u32, const joinx::Range&) {}
    __device__ static void compact_move(const Args& m, Smem&, u32 buf, u32 nb, const joinx::Range& rg, u32 Spn,
                                        const u32* ranks, const u32*) {
        const u16* src = col(m, buf);
        u16* dst = col(m, nb);
        const u32 R = rg.hi - rg.lo;
        for (u32 i = 0; i < m.ncol; i++) {
            for (u32 x = threadIdx.x; x < R; x += kThreads) {
                const u32 r = ranks[x];
                if (r != kNone) dst[(size_t)i * Spn + r] = ld_cg_u16(src + (size_t)i * rg.Sp + rg.lo + x);
            }
        }
    }
    __device__ static void after_compact(const Args&, Smem&, u32, const joinx::Range&) {}
};

template struct IndelDense<true>;
template struct IndelDense<false>;

// ---------------------------------------------------------------------------
// Allele bitsets (integer path).  Row (s, a) of Bits holds one bit per slot:
// set when the slot's cell carries allele code a+2 at site s.  A query's
// score for 32 slots at once is the weighted count, over its edited sites, of
// set bits in the rows of its own alleles; the counts are kept bit-sliced
// (plane k = bit k of every slot's count) so adding a 32-slot word costs a
// few logic operations.  The integer path guarantees every score <= 2048.

constexpr int kPlanes = 12;
constexpr u32 kBitsAlign = 128;      // slots: 4 bitset words, one 16-byte copy
constexpr u32 kStageWords = 14336;   // 56 KB of staged bitset words per round (325 entries of 44 words)

// c += x * w in bit-sliced form (w <= 2048)
__device__ __forceinline__ void vadd(u32 (&c)[kPlanes], u32 x, u32 w) {
    if (!x) return;
    if (w == 1u) {
        u32 carry = x;
#pragma unroll
        for (int k = 0; k < kPlanes; k++) {
            const u32 t = c[k] & carry;
            c[k] ^= carry;
            carry = t;
            if (!carry) break;
        }
        return;
    }
    while (w) {
        const int k0 = __ffs(w) - 1;
        w &= w - 1;
        u32 carry = x;
#pragma unroll
        for (int k = 0; k < kPlanes; k++) {
            if (k < k0) continue;
            const u32 t = c[k] & carry;
            c[k] ^= carry;
            carry = t;
            if (!carry) break;
        }
    }
}

// c += x0 + ... + x7 (unit weights) in bit-sliced form: a carry-save adder
// tree reduces the eight words to a 4-bit per-slot sum (26 logic operations),
// which one ripple adds into the planes; about 7.5 operations per word where
// vadd's carry chain costs several times that.
__device__ __forceinline__ void fa(u32 a, u32 b, u32 c, u32& s, u32& cy) {
    const u32 u = a ^ b;
    s = u ^ c;
    cy = (a & b) | (u & c);
}
__device__ __forceinline__ void vadd8(u32 (&c)[kPlanes], const u32 (&x)[8]) {
    u32 s0, c0, s1, c1, s2, c2, s4, c4;
    fa(x[0], x[1], x[2], s0, c0);
    fa(x[3], x[4], x[5], s1, c1);
    fa(s0, s1, x[6], s2, c2);
    const u32 b0 = s2 ^ x[7], c3 = s2 & x[7];   // weight 1, carry of weight 2
    fa(c0, c1, c2, s4, c4);                       // weight 2 and 4
    const u32 b1 = s4 ^ c3, c5 = s4 & c3;         // weight 2, carry of weight 4
    const u32 b2 = c4 ^ c5, b3 = c4 & c5;         // weight 4 and 8
    u32 cy = c[0] & b0;
    c[0] ^= b0;
    u32 t;
    t = c[1] ^ b1; const u32 n1 = (c[1] & b1) | (t & cy); c[1] = t ^ cy; cy = n1;
    t = c[2] ^ b2; const u32 n2 = (c[2] & b2) | (t & cy); c[2] = t ^ cy; cy = n2;
    t = c[3] ^ b3; const u32 n3 = (c[3] & b3) | (t & cy); c[3] = t ^ cy; cy = n3;
#pragma unroll
    for (int k = 4; k < kPlanes; k++) {
        const u32 n = c[k] & cy;
        c[k] ^= cy;
        cy = n;
    }
}

__device__ __forceinline__ void vsum(u32 (&a)[kPlanes], const u32* b) {
    u32 carry = 0;
#pragma unroll
    for (int k = 0; k < kPlanes; k++) {
        const u32 x = a[k], y = b[k];
        a[k] = x ^ y ^ carry;
        carry = (x & y) | (carry & (x ^ y));
    }
}

__device__ __forceinline__ u32 vget(const u32* p, u32 j) {
    u32 v = 0;
#pragma unroll
    for (int k = 0; k < kPlanes; k++) v |= ((p[k] >> j) & 1u) << k;
    return v;
}

// Bits[row][w] for the tips: one warp per (site, word), lanes = the word's 32
// slots; every distinct allele among them gets one store of its lane mask.
__global__ void k_build_bits(const u16* __restrict__ nodeRow, u32 ntip, u32 ncol, u32 ncolP, u32 nState, u32 Wd,
                             u32* __restrict__ bits) {
    __shared__ u16 tile[32][33];
    const u32 w = blockIdx.x, s0 = blockIdx.y * 32;
    for (u32 r = threadIdx.y; r < 32; r += blockDim.y) {
        const u32 slot = w * 32 + r, s = s0 + threadIdx.x;
        tile[r][threadIdx.x] = (slot < ntip && s < ncol) ? nodeRow[(size_t)slot * ncolP + s] : (u16)0;
    }
    __syncthreads();
    for (u32 y = threadIdx.y; y < 32; y += blockDim.y) {
        const u32 s = s0 + y;
        if (s >= ncol) break;
        const u32 code = tile[threadIdx.x][y];
        const u32 mask = __match_any_sync(0xFFFFFFFFu, code);
        if (code > 1 && (__ffs(mask) - 1) == (int)threadIdx.x)
            bits[((size_t)s * nState + (code - 2)) * Wd + w] = mask;
    }
}

struct InitBitsArgs {
    u32 ntip, ncol, nState, Wd;
    int unitW;
    const u32* bits;
    const u32* eSC;
    const u16* eW;
    const u32* eLen;
    const u64* chunkStart;
    u32 nChunks;
    u64 nTiles;
    unsigned long long* tileCounter;
    unsigned long long* initKey;
};

// Initial local maxima with the bitsets: each 128-thread group takes its own
// (4096-candidate chunk, query) tiles, one 32-slot word per thread.
__global__ void __launch_bounds__(kThreads) k_init_bits(InitBitsArgs a) {
    __shared__ unsigned long long s_tile[4];
    __shared__ u64 red[16];
    const u32 g = threadIdx.x >> 7, t = threadIdx.x & 127, lane = threadIdx.x & 31;
    for (;;) {
        if (t == 0) s_tile[g] = atomicAdd(a.tileCounter, 1ull);
        asm volatile("bar.sync %0, 128;" ::"r"(1 + g));
        const u64 tile = s_tile[g];
        asm volatile("bar.sync %0, 128;" ::"r"(1 + g));
        if (tile >= a.nTiles) break;
        u32 k = 0;
        while (k + 1 < a.nChunks && a.chunkStart[k + 1] <= tile) k++;
        const u32 q = (u32)(tile - a.chunkStart[k]);
        const u32 w = k * 128 + t;
        u64 best = make_key(ORD_F16_NEG1, 0u);
        if (w * 32 < a.ntip && w * 32 + 31 > q) {
            u32 c[kPlanes];
#pragma unroll
            for (int i = 0; i < kPlanes; i++) c[i] = 0u;
            const u32* es = a.eSC + (size_t)q * a.ncol;
            const u16* ew = a.eW + (size_t)q * a.ncol;
            const int nE = (int)a.eLen[q];
            int e = 0;
            for (; e + 7 < nE; e += 8) {
                u32 x[8], wt[8];
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const u32 sc = es[e + i];
                    wt[i] = ew[e + i];
                    x[i] = __ldg(a.bits + ((size_t)(sc & 0xFFFFu) * a.nState + (sc >> 16) - 2) * a.Wd + w);
                }
                if (a.unitW) {
                    vadd8(c, x);
                } else {
#pragma unroll
                    for (int i = 0; i < 8; i++) vadd(c, x[i], wt[i]);
                }
            }
            for (; e < nE; e++) {
                const u32 sc = es[e];
                vadd(c, __ldg(a.bits + ((size_t)(sc & 0xFFFFu) * a.nState + (sc >> 16) - 2) * a.Wd + w), ew[e]);
            }
            u32 any = 0;
#pragma unroll
            for (int i = 0; i < kPlanes; i++) any |= c[i];
            // zero-score slots still compete (score 0 beats the -1 seed)
            for (u32 j = 0; j < 32; j++) {
                const u32 slot = w * 32 + j;
                if (slot <= q || slot >= a.ntip) continue;
                const u32 cnt = ((any >> j) & 1u) ? vget(c, j) : 0u;
                const u64 key = make_key(ord_f16((u16)half_bits_of_int(cnt)), slot);
                best = key > best ? key : best;
            }
        }
        best = warp_max_u64(best);
        if (lane == 0) red[threadIdx.x >> 5] = best;
        asm volatile("bar.sync %0, 128;" ::"r"(1 + g));
        if (t == 0) {
            u64 m = red[g * 4];
            for (int i = 1; i < 4; i++) m = red[g * 4 + i] > m ? red[g * 4 + i] : m;
            atomicMax(a.initKey + q, (unsigned long long)m);
        }
        asm volatile("bar.sync %0, 128;" ::"r"(1 + g));
    }
}

struct IndelBits {
    static constexpr bool kFusedStale = true;  // stale batches share one scan (stale_multi)
    struct Args {
        u32 ncol, ncolP, nState, minSize;
        float minRatio;
        int unitW;
        const u16* Wsel;
        u16* nodeRow;
        u32* bits[2];
        u32 maxBatch;  // query lists kept for a stale batch
    };
    struct Smem {
        u32* eSC;
        u16* eW;
        u16* mrow;
        u16* orow;    // j1's row (the slot's previous occupant)
        u32* planes;  // kThreads x kPlanes
        u64* bbest;   // kMaxBatch: a stale batch's best keys over the passes
        u32* bSC;     // maxBatch x ncol: a stale batch's query lists
        u16* bW;      // maxBatch x ncolW
        u32* bwc;     // kMaxBatch x 33: per-query warp counts of the fused build
        u32* stage;   // kStageWords: bitset words copied for the current round
    };
    __host__ __device__ static size_t engine_smem_bytes(u32 nCTA, u32 Rmax, u32 deathWords = 0, u32 pre = 0) {
        return joinx::engine_smem(nCTA, Rmax, deathWords, pre);
    }
    __host__ __device__ static u32 ncolW(u32 ncol) { return (ncol + 7u) & ~7u; }
    __host__ static size_t model_smem_bytes(const Args& m) {
        return sizeof(u32) * kThreads * kPlanes + sizeof(u32) * kStageWords + sizeof(u64) * joinx::kMaxBatch +
               sizeof(u32) * m.ncol +
               sizeof(u32) * (size_t)m.maxBatch * m.ncol + sizeof(u32) * joinx::kMaxBatch * 33 +
               sizeof(u16) * (ncolW(m.ncol) * (1 + (size_t)m.maxBatch) + 2 * m.ncolP) + 16;
    }
    // bytes of one more query list in a stale batch
    __host__ static size_t batch_list_bytes(u32 ncol) { return sizeof(u32) * ncol + sizeof(u16) * ncolW(ncol); }
    __device__ static void carve_smem(const Args& m, unsigned char* p, Smem& s) {
        s.planes = reinterpret_cast<u32*>(p);
        s.stage = s.planes + kThreads * kPlanes;
        s.bbest = reinterpret_cast<u64*>(s.stage + kStageWords);
        s.eSC = reinterpret_cast<u32*>(s.bbest + joinx::kMaxBatch);
        s.bSC = s.eSC + m.ncol;
        s.bwc = s.bSC + (size_t)m.maxBatch * m.ncol;
        s.eW = reinterpret_cast<u16*>(s.bwc + joinx::kMaxBatch * 33);
        s.bW = s.eW + ncolW(m.ncol);
        s.mrow = s.bW + (size_t)m.maxBatch * ncolW(m.ncol);
        s.orow = s.mrow + m.ncolP;
    }
    __device__ static u32* bitsOf(const Args& m, u32 buf) { return buf ? m.bits[1] : m.bits[0]; }
    __device__ static int build_stale(const Args& m, Smem& s, u32 j1, u32* wc) {
        return build_indel_query(m.ncol, m.ncolP, m.unitW, m.Wsel, m.nodeRow + (size_t)j1 * m.ncolP, nullptr, 0,
                                 nullptr, nullptr, s.eSC, s.eW, wc);
    }
    __device__ static int build_join(const Args& m, Smem& s, u32 j1, u32 j2, u32 s1, u32 s2, u32* wc) {
        int mode;
        if (s1 < m.minSize && __uint2float_rn(s1) * m.minRatio < __uint2float_rn(s2)) mode = 1;
        else if (s2 < m.minSize && __uint2float_rn(s2) * m.minRatio < __uint2float_rn(s1)) mode = 2;
        else mode = 3;
        // j1's row is left in orow for store_slot by the same loads
        return build_indel_query(m.ncol, m.ncolP, m.unitW, m.Wsel, m.nodeRow + (size_t)j1 * m.ncolP,
                                 m.nodeRow + (size_t)j2 * m.ncolP, mode, s.mrow, s.orow, s.eSC, s.eW, wc);
    }
    // slice `part` of `nparts` of the new node's row (the engine writes it whole)
    __device__ static void store_node(const Args& m, Smem& s, u32 newNode, u32 part, u32 nparts) {
        u16* dst = m.nodeRow + (size_t)newNode * m.ncolP;
        const u32 per = (m.ncolP + nparts - 1) / nparts, i1 = min(m.ncolP, (part + 1) * per);
        for (u32 i = part * per + threadIdx.x; i < i1; i += kThreads) dst[i] = s.mrow[i];
    }
    // the new node replaces j1 in slot c1: flip c1's bit in the rows of slice
    // `part` of `nparts` of the sites where the two states differ (the engine
    // gives all of them to c1's owner; fire-and-forget reductions on single
    // bits; c1 is skipped by this phase's scans, and the next phase reads the
    // words after the grid barrier)
    __device__ static void store_slot(const Args& m, Smem& s, u32 buf, const joinx::Range& rg, u32 c1, u32 part,
                                      u32 nparts) {
        u32* B = bitsOf(m, buf);
        const u32 Wd = rg.Sp / 32, word = c1 >> 5, bit = 1u << (c1 & 31);
        const u32 per = (m.ncol + nparts - 1) / nparts, i1 = min(m.ncol, (part + 1) * per);
        for (u32 i = part * per + threadIdx.x; i < i1; i += kThreads) {
            const u32 o = s.orow[i], n = s.mrow[i];
            if (o == n) continue;
            if (o > 1) atomicAnd(B + ((size_t)i * m.nState + o - 2) * Wd + word, ~bit);
            if (n > 1) atomicOr(B + ((size_t)i * m.nState + n - 2) * Wd + word, bit);
        }
    }
    __host__ __device__ static u32 pass_cap(const Args&, u32 R) {
        const u32 r = (R + 31u) & ~31u;
        return r < 4096u ? r : 4096u;
    }

    // Bit-sliced counts of nq queries over the bitset words [w0, w0 + Wc) of
    // this CTA.  Query q's entries are lists eSC/eW + q * stride (nE[q] of
    // them); the queries' entries form one sequence that is staged in shared
    // memory round by round: every thread issues its 16-byte cp.async copies
    // of the round's (entry, 4 words) pieces, so a round costs one trip to
    // L2/HBM whatever the number of queries and holds no data in registers.
    // Thread (q, g, t) of set q (setSize threads), group g < F of TG threads,
    // then adds word t of entries g, g + F, ... of query q into c.
    __device__ static void staged_counts(const Args& m, Smem& s, const u32* B, u32 Wd, u32 w0, u32 Wc, u32 nq,
                                         const u32* eSC0, const u16* eW0, u32 strideSC, u32 strideW, const int* nEq,
                                         u32 setSize, u32 TG, u32 F, u32 (&c)[kPlanes]) {
        const u32 Wc4 = (Wc + 3u) & ~3u, cpe = Wc4 / 4;  // 16-byte pieces per entry
        const u32 q = threadIdx.x / setSize, ts = threadIdx.x % setSize;
        const u32 g = ts / TG, t = ts % TG;
        __shared__ u32 off[joinx::kMaxBatch + 1];  // query q's entries start at off[q]
        if (threadIdx.x == 0) {
            off[0] = 0;
            for (u32 i = 0; i < nq; i++) off[i + 1] = off[i] + (u32)nEq[i];
        }
        __syncthreads();
        const u32 total = off[nq];
        const u32 per = kStageWords / Wc4;  // entries per round
        const u32 myOff = q < nq ? off[q] : 0u, myN = q < nq ? (u32)nEq[q] : 0u;
        const u16* eWq = eW0 + (size_t)(q < nq ? q : 0) * strideW;
        const bool active = q < nq && g < F && t < Wc;
        // copy mapping: lane = (entry j of the warp's epw, piece k); no division in the loop
        const u32 lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        const u32 epw = 32 / cpe, jl = lane / cpe, kl = lane % cpe;
        const bool copier = jl < epw;
        // copies of entries [a, b) of the round starting at r0
        auto copy_range = [&](u32 r0, u32 a, u32 b) {
            if (!copier) return;
            u32 qq = 0;
            for (u32 ce = a + wid * epw + jl; ce < b; ce += (kThreads / 32) * epw) {
                while (qq + 1 < nq && ce >= off[qq + 1]) qq++;
                const u32 sc = eSC0[(size_t)qq * strideSC + (ce - off[qq])];
                cp_async16(s.stage + (size_t)(ce - r0) * Wc4 + 4 * kl,
                           B + ((size_t)(sc & 0xFFFFu) * m.nState + (sc >> 16) - 2) * Wd + w0 + 4 * kl);
            }
        };
        // this thread's additions from the staged entries [a, b)
        auto add_range = [&](u32 r0, u32 a, u32 b) {
            if (!active) return;
            const u32 lo = max(a, myOff) - myOff, hi = min(b, myOff + myN);
            if (myOff + lo >= hi) return;
            u32 e = lo + (g + F - lo % F) % F;  // first entry >= lo of this group
            const u32 end = hi - myOff;
            if (m.unitW) {
                for (; e < end; e += 8 * F) {  // the last group of 8 is padded with zero words
                    u32 x[8];
#pragma unroll
                    for (int j = 0; j < 8; j++)
                        x[j] = e + j * F < end ? s.stage[(size_t)(myOff + e + j * F - r0) * Wc4 + t] : 0u;
                    vadd8(c, x);
                }
            }
            for (; e + 3 * F < end; e += 4 * F) {
                u32 x[4], wt[4];
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    x[j] = s.stage[(size_t)(myOff + e + j * F - r0) * Wc4 + t];
                    wt[j] = eWq[e + j * F];
                }
#pragma unroll
                for (int j = 0; j < 4; j++) vadd(c, x[j], wt[j]);
            }
            for (; e < end; e += F) vadd(c, s.stage[(size_t)(myOff + e - r0) * Wc4 + t], eWq[e]);
        };
        // each round in two halves: the first half is added while the second is in flight
        for (u32 r0 = 0; r0 < total; r0 += per) {
            const u32 r1 = min(total, r0 + per), rm = r0 + (r1 - r0 + 1) / 2;
            copy_range(r0, r0, rm);
            cp_async_commit();
            copy_range(r0, rm, r1);
            cp_async_commit();
            cp_async_wait_group<1>();
            __syncthreads();
            joinx::prof_mark(joinx::PROF_SC_COPY);
            add_range(r0, r0, rm);
            cp_async_wait_group<0>();
            __syncthreads();
            add_range(r0, rm, r1);
            __syncthreads();  // the next round overwrites the stage
            joinx::prof_mark(joinx::PROF_SC_ACC);
        }
        // copies the caller issued before (slot prefetch) are complete even
        // when there was no entry to stage; the caller's next barrier
        // publishes them
        cp_async_wait_all();
    }

    // Sums the F groups' counters of word t (groups of TG threads, planes
    // area P) into P[t] by a tree of ceil(log2 F) rounds; F need not be a
    // power of two.  Block-wide barriers: every set of a CTA calls it with
    // the same F.
    __device__ static void reduce_groups(u32 (&c)[kPlanes], u32* P, u32 g, u32 t, u32 TG, u32 F, bool live) {
        for (u32 Fl = F; Fl > 1;) {
            const u32 h = (Fl + 1) / 2;
            if (live && g >= h && g < Fl) {
#pragma unroll
                for (int i = 0; i < kPlanes; i++) P[((g - h) * TG + t) * kPlanes + i] = c[i];
            }
            __syncthreads();
            if (live && g < Fl - h) vsum(c, P + (g * TG + t) * kPlanes);
            __syncthreads();
            Fl = h;
        }
        if (live && g == 0) {
#pragma unroll
            for (int i = 0; i < kPlanes; i++) P[t * kPlanes + i] = c[i];
        }
        __syncthreads();
    }

    __device__ static void score_pass(const Args& m, Smem& s, u32 buf, const joinx::Range& rg, u32 base, u32 cap,
                                      int nE, u32* ordOut) {
        const u32 T = cap / 32;
        const u32 Wd = rg.Sp / 32;
        const u32 Wc = min(T, (rg.hi - base + 31u) / 32u);
        // groups of exactly Wc threads (one per word), as many as fit, at most 16
        const u32 TG = Wc, F = min(kThreads / TG, 16u);
        const u32 g = threadIdx.x / TG, t = threadIdx.x % TG;
        u32 c[kPlanes];
#pragma unroll
        for (int i = 0; i < kPlanes; i++) c[i] = 0u;
        __shared__ int s_nE1;  // read by thread 0 before staged_counts' first barrier, by all after it
        if (threadIdx.x == 0) s_nE1 = nE;
        staged_counts(m, s, bitsOf(m, buf), Wd, base / 32, Wc, 1, s.eSC, s.eW, 0, 0, &s_nE1, kThreads, TG, F, c);
        reduce_groups(c, s.planes, g, t, TG, F, g < F);
        for (u32 x = threadIdx.x; x < cap && base + x < rg.hi; x += kThreads) {
            const u32 cnt = vget(s.planes + (x >> 5) * kPlanes, x & 31);
            ordOut[x] = ord_f16((u16)half_bits_of_int(cnt));
        }
        __syncthreads();
        joinx::prof_mark(joinx::PROF_SC_RED);
    }
    // Query lists of nq stale rows at once: the rows are staged in shared
    // memory (in the planes area, unused until the scan) by one round of
    // 16-byte loads, then each list is compacted with a block prefix sum; the
    // nq sums share two block barriers.  List q goes to bSC/bW + q.  Needs
    // nq * ncolP u16 <= the planes area (build_multi_fits).
    __device__ static bool build_multi_fits(const Args& m, u32 nq) {
        return (size_t)nq * m.ncolP * sizeof(u16) <= sizeof(u32) * kThreads * kPlanes;
    }
    // Issues the asynchronous copies of the nq rows into the staging area.
    __device__ static void stage_rows_async(const Args& m, Smem& s, u32 nq, const joinx::BlockRec* rows) {
        u16* stage = reinterpret_cast<u16*>(s.planes);
        const u32 v16 = m.ncolP / 8;  // 16-byte words per row (ncolP is a multiple of 8)
        for (u32 i = threadIdx.x; i < nq * v16; i += kThreads) {
            const u32 q = i / v16, x = i % v16;
            cp_async16(stage + (size_t)q * m.ncolP + 8 * x, m.nodeRow + (size_t)key_node(rows[q].key) * m.ncolP + 8 * x);
        }
    }
    // Expects the rows staged (stage_rows_async, then wait and a barrier).
    __device__ static void build_multi(const Args& m, Smem& s, u32 nq, int* nEout) {
        const u32 lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        const u16* stage = reinterpret_cast<const u16*>(s.planes);
        const u32 per = (m.ncol + kThreads - 1) / kThreads;
        const u32 s0 = threadIdx.x * per, s1 = min(s0 + per, m.ncol);
        for (u32 q = 0; q < nq; q++) {
            const u16* row = stage + (size_t)q * m.ncolP;
            u32 c = 0;
            for (u32 x = s0; x < s1; x++) c += row[x] > 1;
            u32 v = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const u32 n = __shfl_up_sync(0xFFFFFFFFu, v, o);
                if (lane >= (u32)o) v += n;
            }
            if (lane == 31) s.bwc[q * 33 + wid] = v;
        }
        __syncthreads();
        // warp q: exclusive offsets of the 16 warps' counts of query q
        if (wid < nq) {
            const u32 v = lane < kThreads / 32 ? s.bwc[wid * 33 + lane] : 0u;
            u32 wi = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const u32 n = __shfl_up_sync(0xFFFFFFFFu, wi, o);
                if (lane >= (u32)o) wi += n;
            }
            __syncwarp();
            if (lane < kThreads / 32) s.bwc[wid * 33 + 16 + lane] = wi - v;
            if (lane == kThreads / 32 - 1) s.bwc[wid * 33 + 32] = wi;
        }
        __syncthreads();
        for (u32 q = 0; q < nq; q++) {
            const u16* row = stage + (size_t)q * m.ncolP;
            // this thread's offset: its warp's offset plus the earlier lanes' counts
            u32 c = 0;
            for (u32 x = s0; x < s1; x++) c += row[x] > 1;
            u32 v = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const u32 n = __shfl_up_sync(0xFFFFFFFFu, v, o);
                if (lane >= (u32)o) v += n;
            }
            u32 pos = s.bwc[q * 33 + 16 + wid] + v - c;
            u32* eSC = s.bSC + (size_t)q * m.ncol;
            u16* eW = s.bW + (size_t)q * ncolW(m.ncol);
            for (u32 x = s0; x < s1; x++) {
                const u32 code = row[x];
                if (code > 1) {
                    eSC[pos] = x | (code << 16);
                    eW[pos] = m.unitW ? (u16)1 : m.Wsel[(size_t)(code - 2) * m.ncol + x];
                    pos++;
                }
            }
        }
        if (threadIdx.x < nq) nEout[threadIdx.x] = (int)s.bwc[threadIdx.x * 33 + 32];
        __syncthreads();
    }

    // Rescans of nq stale rows in one pass over the allele bitsets.  The CTA
    // splits into nq thread sets (512/2^ceil(log2 nq) threads each); in set q
    // thread (g, t) adds query q's entries g, g+F, ... for the 32 slots of
    // word t, so all nq queries' bitset loads are in flight together.  The F
    // groups' bit-sliced counters are summed in shared memory and best[q]
    // gets the top (score, node) key over the live slots other than row q's.
    __device__ static void stale_multi(const Args& m, Smem& s, u32 buf, const joinx::Range& rg, const u32* sn, u32 nq,
                                       const joinx::BlockRec* rows, u64* best, int* nEout, u32* snCache, u64* red,
                                       u32* wc) {
        const u32 nqP = nq <= 1 ? 1u : (nq <= 2 ? 2u : (nq <= 4 ? 4u : 8u));
        const u32 setSize = kThreads / nqP;
        const u32 capMax = min(setSize * 32u, joinx::kMaxCap);
        // the first pass's slot nodes and the staged rows share one round trip
        const u32 cap0 = min(capMax, (rg.hi - rg.lo + 31u) & ~31u);
        if (rg.lo < rg.hi)
            for (u32 i = threadIdx.x; i < cap0 / 4; i += kThreads) cp_async16(snCache + 4 * i, sn + rg.lo + 4 * i);
        const bool fused = build_multi_fits(m, nq);
        if (fused) stage_rows_async(m, s, nq, rows);
        cp_async_wait_all();
        __syncthreads();
        if (fused) {
            build_multi(m, s, nq, nEout);
        } else {
            for (u32 q = 0; q < nq; q++) {
                const int n = build_indel_query(m.ncol, m.ncolP, m.unitW, m.Wsel,
                                                m.nodeRow + (size_t)key_node(rows[q].key) * m.ncolP, nullptr, 0,
                                                nullptr, nullptr, s.bSC + (size_t)q * m.ncol,
                                                s.bW + (size_t)q * ncolW(m.ncol), wc);
                if (threadIdx.x == 0) nEout[q] = n;
            }
            __syncthreads();
        }
        const u32 q = threadIdx.x / setSize, ts = threadIdx.x % setSize;
        const u32 lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        const u32 Wd = rg.Sp / 32;
        const u32* B = bitsOf(m, buf);
        const u32 myRow = q < nq ? rows[q].slot : kNone;
        if (threadIdx.x < joinx::kMaxBatch) s.bbest[threadIdx.x] = 0ull;
        for (u32 base = rg.lo; base < rg.hi; base += capMax) {
            const u32 cap = min(capMax, (rg.hi - base + 31u) & ~31u);
            const u32 Wc = cap / 32;
            if (base != rg.lo) {  // later passes copy their slot nodes here
                __syncthreads();
                for (u32 i = threadIdx.x; i < cap / 4; i += kThreads) cp_async16(snCache + 4 * i, sn + base + 4 * i);
                cp_async_wait_all();
                __syncthreads();
            }
            // groups of exactly Wc threads (one per word), at most 16 per set
            const u32 TG = Wc, F = min(setSize / TG, 16u);
            const u32 g = ts / TG, t = ts % TG;
            u32 c[kPlanes];
#pragma unroll
            for (int i = 0; i < kPlanes; i++) c[i] = 0u;
            staged_counts(m, s, B, Wd, base / 32, Wc, nq, s.bSC, s.bW, m.ncol, ncolW(m.ncol), nEout, setSize, TG, F,
                          c);
            // sum the F groups' counters of (q, t) into group 0's entry
            u32* P = s.planes + (size_t)(q < nqP ? q : 0) * setSize * kPlanes;
            reduce_groups(c, P, g, t, TG, F, q < nq && g < F);
            // best key of query q over this pass's live slots
            u64 bk = 0ull;
            if (q < nq) {
                for (u32 x = ts; x < cap; x += setSize) {
                    const u32 slot = base + x, node = snCache[x];
                    if (slot >= rg.hi || node == joinx::kDead || slot == myRow) continue;
                    const u32 cnt = vget(P + (x >> 5) * kPlanes, x & 31);
                    const u64 key = make_key(ord_f16((u16)half_bits_of_int(cnt)), node);
                    bk = key > bk ? key : bk;
                }
            }
            bk = warp_max_u64(bk);
            if (lane == 0) red[wid] = bk;
            __syncthreads();
            if (threadIdx.x < nq) {
                const u32 w0 = threadIdx.x * (setSize / 32), w1 = w0 + setSize / 32;
                u64 b2 = s.bbest[threadIdx.x];
                for (u32 i = w0; i < w1; i++) b2 = red[i] > b2 ? red[i] : b2;
                s.bbest[threadIdx.x] = b2;
            }
            __syncthreads();
        }
        if (threadIdx.x < nq) best[threadIdx.x] = s.bbest[threadIdx.x];
        __syncthreads();
    }
    // C1: clear this CTA's words of the new layout in every row
    __device__ static void compact_prepare(const Args& m, Smem&, u32 nb, const joinx::Range& nr) {
        u32* B = bitsOf(m, nb);
        const u32 Wdn = nr.Sp / 32, w0 = nr.lo / 32, w1 = (nr.hi + 31) / 32;
        if (w1 <= w0) return;
        const u32 nw = w1 - w0;
        const size_t rows = (size_t)m.ncol * m.nState;
        for (size_t i = threadIdx.x; i < rows * nw; i += kThreads) {
            const size_t row = i / nw;
            B[row * Wdn + w0 + (u32)(i % nw)] = 0u;
        }
    }
    // C2: set the bits of every live slot of this CTA at its new position
    // (words may belong to another CTA in the new layout, hence atomics)
    __device__ static void compact_move(const Args& m, Smem&, u32, u32 nb, const joinx::Range& rg, u32 Spn,
                                        const u32* ranks, const u32* slotNodeOld) {
        u32* B = bitsOf(m, nb);
        const u32 Wdn = Spn / 32;
        const u32 R = rg.hi - rg.lo;
        const u32 lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        for (u32 x = wid; x < R; x += kThreads / 32) {
            const u32 r = ranks[x];
            if (r == kNone) continue;
            const u32 node = ld_cg_u32(slotNodeOld + rg.lo + x);
            const u16* row = m.nodeRow + (size_t)node * m.ncolP;
            const u32 word = r >> 5, bit = 1u << (r & 31);
            for (u32 i = lane; i < m.ncol; i += 32) {
                const u32 code = ld_cg_u16(row + i);
                if (code > 1) atomicOr(B + ((size_t)i * m.nState + code - 2) * Wdn + word, bit);
            }
        }
    }
    __device__ static void after_compact(const Args&, Smem&, u32, const joinx::Range&) {}
};

// state_out[r] = nodeRow[order[r]] widened to u32
__global__ void k_gather(const u16* __restrict__ nodeRow, u32 ncol, u32 ncolP, const u32* __restrict__ order,
                         u32 nrows, u32* __restrict__ out) {
    const u32 r = blockIdx.x;
    if (r >= nrows) return;
    const u16* src = nodeRow + (size_t)order[r] * ncolP;
    u32* dst = out + (size_t)r * ncol;
    for (u32 s = threadIdx.x; s < ncol; s += blockDim.x) dst[s] = src[s];
}

}  // namespace indel

// ---------------------------------------------------------------------------
// host side

using namespace indel;

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

// Device buffers of one indel join (shared by the allocating and the
// zero-allocation entry points).
struct IndelBuffers {
    u16* Wsel; u16* nodeRow; u16* colT0; u16* colT1; u32* bits0; u32* bits1; size_t bitsWords; u32* lm[6];
    u32* node2slot; u32* nodeDeath; u32* nodeSize; u32* rawEdge;
    u32* eSC; u16* eW; u32* eLen; unsigned long long* initKey;
    joinx::BlockRec* pub; u32* pubCnt; u64* partial; u32* counts; u32* flags; int* jerr; int* prepErr;
    unsigned long long* tileCounter; u64* chunkStart; unsigned long long* stats; u32* tipSize;
};

// Bytes of the two allele-bitset buffers for the bitset scan.
static size_t bits_bytes(u32 ntip, u32 ncol, u32 nState) {
    const size_t Wd = ((size_t)ntip + kBitsAlign - 1) / kBitsAlign * (kBitsAlign / 32);
    return 2 * (size_t)ncol * nState * Wd * sizeof(u32);
}

static IndelBuffers carve_indel(Carve& c, u32 ntip, u32 ncol, u32 nState, u32 nCTA, u32 nChunks, bool useBits) {
    const u32 nnode = 2 * ntip - 1, nedge = 2 * ntip - 2;
    // the bitset scan copies 16-byte pieces of bitset rows: slot ranges and
    // row strides are multiples of 128 slots (kBitsAlign)
    const u32 ncolP = (ncol + 7u) & ~7u, Sp = useBits ? (ntip + kBitsAlign - 1) / kBitsAlign * kBitsAlign
                                                      : (ntip + 31u) & ~31u;
    const size_t nw = (size_t)nState * ncol;
    IndelBuffers l;
    l.Wsel = c.take<u16>(nw ? nw : 1);
    l.nodeRow = c.take<u16>((size_t)nnode * ncolP);
    l.colT0 = c.take<u16>(useBits ? 0 : (size_t)ncol * Sp);
    l.colT1 = c.take<u16>(useBits ? 0 : (size_t)ncol * Sp);
    l.bitsWords = useBits ? (size_t)ncol * nState * (Sp / 32) : 0;
    l.bits0 = c.take<u32>(l.bitsWords);
    l.bits1 = c.take<u32>(l.bitsWords);
    for (int i = 0; i < 6; i++) l.lm[i] = c.take<u32>(Sp);
    l.node2slot = c.take<u32>(nnode);
    l.nodeDeath = c.take<u32>(nnode);
    l.nodeSize = c.take<u32>(nnode);
    l.rawEdge = c.take<u32>((size_t)2 * nedge + 2);
    l.eSC = c.take<u32>((size_t)ntip * ncol);
    l.eW = c.take<u16>((size_t)ntip * ncol);
    l.eLen = c.take<u32>(ntip);
    l.initKey = c.take<unsigned long long>(ntip);
    l.pub = c.take<joinx::BlockRec>(4 * nCTA);
    l.pubCnt = c.take<u32>(2 * nCTA);
    l.partial = c.take<u64>((size_t)2 * nCTA * joinx::kMaxBatch);
    l.counts = c.take<u32>(nCTA);
    l.flags = c.take<u32>(16 * nCTA);
    l.jerr = c.take<int>(1);
    l.prepErr = c.take<int>(1);
    l.tileCounter = c.take<unsigned long long>(1);
    l.chunkStart = c.take<u64>(nChunks + 1);
    l.stats = c.take<unsigned long long>(8 + joinx::PROF_N);
    l.tipSize = c.take<u32>(ntip);
    return l;
}

static void chunk_table(u32 ntip, u32 nChunks, u64* chunkStart) {
    chunkStart[0] = 0;
    for (u32 k = 0; k < nChunks; k++) {
        const u64 end = std::min<u64>((u64)(k + 1) * kCap, ntip);
        chunkStart[k + 1] = chunkStart[k] + (end >= 1 ? end - 1 : 0);
    }
}

// Launches the persistent join of model M after fitting its shared memory
// to the device: first fewer query lists per stale batch (when the model
// keeps them, *batch), then no joined-node bitmap (the engine then reads
// node deaths from global memory).
template <class M>
static int launch_join_fitted(joinx::Common& c, typename M::Args& m, u32* batch, u32 nCTA, cudaStream_t st) {
    int smemMax = 0, dev = 0;
    CASPHY_CUDA_TRY(cudaGetDevice(&dev));
    CASPHY_CUDA_TRY(cudaDeviceGetAttribute(&smemMax, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t lim = (size_t)smemMax - 4096;  // the kernel's static shared memory
    auto need = [&] {
        return M::engine_smem_bytes(nCTA, c.Rmax, c.deathWords, c.preSlots) + M::model_smem_bytes(m);
    };
    // shared memory goes first to the joined-node bitmap, then to slot
    // prefetch (models that stage their scan, one pass per range), then to
    // stale batches beyond 4 rows, then to the rest of the batches
    c.preSlots = M::kFusedStale && c.Rmax <= M::pass_cap(m, c.Rmax) ? 1u : 0u;
    const u32 want = batch ? *batch : 1u;
    if (batch) {
        while (*batch > 4 && need() > lim) (*batch)--;
        if (need() > lim) {
            c.preSlots = 0;
            *batch = want;
        }
        while (*batch > 1 && need() > lim) (*batch)--;
        c.maxBatch = *batch;
    } else if (need() > lim) {
        c.preSlots = 0;
    }
    if (need() > lim) c.deathWords = 0;
    const size_t smem = need();
    void* fn = (void*)joinx::k_join<M>;
    CASPHY_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    void* args[] = {&c, &m};
    CASPHY_CUDA_TRY(cudaLaunchCooperativeKernel(fn, dim3(nCTA), dim3(kThreads), args, smem, st));
    return CASPHY_OK;
}

// Launches prep, initial scan and the persistent join.  Assumes Wsel,
// tipSize and chunkStart are already on the device; clears everything the
// kernels expect at zero.  Returns the number of kernels launched.
static int launch_indel(const IndelBuffers& L, u32 ntip, u32 ncol, u32 nState, const u32* codes, bool intPath,
                        bool unitW, bool useBits, u32 minSize, float minRatio, u32 nSM, u32 nChunks, u64 nTiles,
                        cudaStream_t st, cudaEvent_t evInit0, cudaEvent_t evInit1, int* launches) {
    const u32 nnode = 2 * ntip - 1;
    // slot stride: bitset words need multiples of 32 slots, the u16 column
    // scan multiples of 8 (one 16-byte load); the engine uses the same rule
    const u32 align = useBits ? kBitsAlign : 8u;
    const u32 ncolP = (ncol + 7u) & ~7u, Sp = (ntip + align - 1) / align * align;
    const u32 nCTA = nSM;
    CASPHY_CUDA_TRY(cudaMemsetAsync(L.prepErr, 0, sizeof(int), st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(L.jerr, 0, sizeof(int), st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(L.flags, 0, sizeof(u32) * 16 * nCTA, st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(L.tileCounter, 0, sizeof(unsigned long long), st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(L.stats, 0, sizeof(unsigned long long) * 8, st));
    PrepArgs pa{ntip, ncol, ncolP, nState, Sp, codes, L.Wsel, intPath ? 0x7FFFu : 0xFFFFu,
                L.nodeRow, L.eSC, L.eW, L.eLen, L.prepErr};
    k_prep_rows<<<(ntip + 7) / 8, 256, 0, st>>>(pa);
    if (useBits) {
        CASPHY_CUDA_TRY(cudaMemsetAsync(L.bits0, 0, sizeof(u32) * L.bitsWords, st));
        k_build_bits<<<dim3(Sp / 32, (ncol + 31) / 32), dim3(32, 8), 0, st>>>(L.nodeRow, ntip, ncol, ncolP, nState,
                                                                                Sp / 32, L.bits0);
    } else {
        k_transpose<<<dim3((Sp + 31) / 32, (ncol + 31) / 32), dim3(32, 8), 0, st>>>(L.nodeRow, ntip, ncol, ncolP,
                                                                                      Sp, L.colT0);
    }
    joinx::k_fill_u64<<<(ntip + 255) / 256, 256, 0, st>>>(L.initKey, ntip,
                                                           ((u64)ORD_F16_NEG1 << 32) | 0xFFFFFFFFull);
    int n = 3;
    if (evInit0) CASPHY_CUDA_TRY(cudaEventRecord(evInit0, st));
    InitArgs ia{ntip, ncol, Sp, L.colT0, L.eSC, L.eW, L.eLen, L.chunkStart, nChunks, nTiles, L.tileCounter, L.initKey};
    int perSM = 0;
    if (useBits) {
        InitBitsArgs ib{ntip, ncol, nState, Sp / 32, unitW ? 1 : 0, L.bits0, L.eSC, L.eW, L.eLen, L.chunkStart, nChunks, nTiles,
                        L.tileCounter, L.initKey};
        CASPHY_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_init_bits, kThreads, 0));
        k_init_bits<<<nSM * std::max(perSM, 1), kThreads, 0, st>>>(ib);
    } else if (intPath) {
        CASPHY_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_init_scan<true>, kThreads, 0));
        k_init_scan<true><<<nSM * std::max(perSM, 1), kThreads, 0, st>>>(ia);
    } else {
        CASPHY_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_init_scan<false>, kThreads, 0));
        k_init_scan<false><<<nSM * std::max(perSM, 1), kThreads, 0, st>>>(ia);
    }
    n++;
    if (evInit1) CASPHY_CUDA_TRY(cudaEventRecord(evInit1, st));
    const u32 initN = std::max(Sp, nnode);  // Sp: slots rounded up to 32
    joinx::k_slot_init<<<(initN + 255) / 256, 256, 0, st>>>(ntip, Sp, nnode, L.initKey, ORD_F16_NEG1, L.lm[0],
                                                              L.lm[1], L.lm[2], L.node2slot, L.nodeDeath, L.nodeSize,
                                                              L.tipSize);
    n++;
    joinx::Common c{};
    c.ntip = ntip; c.nnode = nnode; c.nCTA = nCTA; c.align = 8;
    c.lmOrd[0] = L.lm[0]; c.lmIdx[0] = L.lm[1]; c.slotNode[0] = L.lm[2];
    c.lmOrd[1] = L.lm[3]; c.lmIdx[1] = L.lm[4]; c.slotNode[1] = L.lm[5];
    c.node2slot = L.node2slot; c.nodeDeath = L.nodeDeath; c.nodeSize = L.nodeSize; c.rawEdge = L.rawEdge;
    c.pub = L.pub; c.pubCnt = L.pubCnt; c.partial = L.partial; c.counts = L.counts; c.flags = L.flags;
    c.err = L.jerr; c.limitNs = 20ull * 1000 * 1000 * 1000; c.statsOut = L.stats;
    c.prof = getenv("CASPHY_PROFILE") ? L.stats + 8 : nullptr;
    c.Rmax = (((ntip + nCTA - 1) / nCTA) + 31u) & ~31u;
    c.ordNeg1 = ORD_F16_NEG1; c.compactMin = 4096; c.compactQ8 = 192; c.bytesPerPairSite = 2000;
    c.maxBatch = joinx::stale_batch_setting();
    c.deathWords = (nnode + 31) / 32;  // 50 KB at 200k cells
    c.needSizes = minSize > 0;         // the minSize / minRatio rule reads node sizes
    if (useBits) {
        using M = IndelBits;
        c.align = kBitsAlign;
        c.Rmax = (((ntip + nCTA - 1) / nCTA) + kBitsAlign - 1) / kBitsAlign * kBitsAlign;
        c.compactQ8 = 128;
        c.bytesPerPairSite = 125;  // one bit per (candidate, query site)
        M::Args m{ncol, ncolP, nState, minSize, minRatio, unitW ? 1 : 0, L.Wsel, L.nodeRow, {L.bits0, L.bits1},
                  c.maxBatch};
        if (int rc = launch_join_fitted<M>(c, m, &m.maxBatch, nCTA, st)) return rc;
    } else if (intPath) {
        using M = IndelDense<true>;
        M::Args m{ncol, ncolP, nState, minSize, minRatio, unitW ? 1 : 0, L.Wsel, L.nodeRow, {L.colT0, L.colT1}};
        if (int rc = launch_join_fitted<M>(c, m, nullptr, nCTA, st)) return rc;
    } else {
        using M = IndelDense<false>;
        M::Args m{ncol, ncolP, nState, minSize, minRatio, 0, L.Wsel, L.nodeRow, {L.colT0, L.colT1}};
        if (int rc = launch_join_fitted<M>(c, m, nullptr, nCTA, st)) return rc;
    }
    n++;
    *launches = n;
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
    const u32 nedge = 2 * ntip - 2, nrows = std::max(ntip - 1, 1u);
    int nSM = 0;
    CASPHY_CUDA_TRY(cudaDeviceGetAttribute(&nSM, cudaDevAttrMultiProcessorCount, ds.dev));
    const u32 nChunks = (ntip + kCap - 1) / kCap;
    // allele-bitset scan on the integer path when the two bitset buffers fit
    // a 48 GiB budget (CASPHY_INDEL_SCAN=dense forces the column scan)
    const char* scanEnv = getenv("CASPHY_INDEL_SCAN");
    bool useBits = intPath && ntip >= 2 && bits_bytes(ntip, ncol, nState) <= (size_t(48) << 30);
    if (scanEnv && !strcmp(scanEnv, "dense")) useBits = false;
    lst.scan_path = useBits ? 1u : 0u;
    Carve cv;
    carve_indel(cv, ntip, ncol, nState, (u32)nSM, nChunks, useBits);
    u32* dCodesCopy = cv.take<u32>(h_codes ? (size_t)ntip * ncol : 0);
    u32* dOrder = cv.take<u32>(nrows);
    u32* dState = cv.take<u32>(h_state_out ? (size_t)nrows * ncol : 0);
    void* base = nullptr;
    rc = ds.reserve(cv.off + 256, &base);
    if (rc) return rc;
    Carve c2;
    c2.base = static_cast<char*>(base);
    const IndelBuffers L = carve_indel(c2, ntip, ncol, nState, (u32)nSM, nChunks, useBits);
    dCodesCopy = c2.take<u32>(h_codes ? (size_t)ntip * ncol : 0);
    dOrder = c2.take<u32>(nrows);
    dState = c2.take<u32>(h_state_out ? (size_t)nrows * ncol : 0);

    cudaEvent_t ev[5];
    for (auto& e : ev) CASPHY_CUDA_TRY(cudaEventCreate(&e));
    CASPHY_CUDA_TRY(cudaEventRecord(ev[0], st));
    const u32* codes = d_codes;
    if (h_codes) {
        CASPHY_CUDA_TRY(cudaMemcpyAsync(dCodesCopy, h_codes, sizeof(u32) * (size_t)ntip * ncol,
                                        cudaMemcpyHostToDevice, st));
        codes = dCodesCopy;
    }
    std::vector<u64> chunkStart(nChunks + 1);
    chunk_table(ntip, nChunks, chunkStart.data());
    CASPHY_CUDA_TRY(cudaMemcpyAsync(L.Wsel, intPath ? wint.data() : hbits.data(), sizeof(u16) * hbits.size(),
                                    cudaMemcpyHostToDevice, st));
    CASPHY_CUDA_TRY(cudaMemcpyAsync(L.tipSize, tipSize, sizeof(u32) * ntip, cudaMemcpyHostToDevice, st));
    CASPHY_CUDA_TRY(cudaMemcpyAsync(L.chunkStart, chunkStart.data(), sizeof(u64) * (nChunks + 1),
                                    cudaMemcpyHostToDevice, st));
    int launches = 0;
    std::vector<u32> order(nrows, 0u);
    unsigned long long hst[8] = {0};
    if (ntip >= 2) {
        rc = launch_indel(L, ntip, ncol, nState, codes, intPath, unitW, useBits, minSize, minRatio, (u32)nSM,
                          nChunks, chunkStart[nChunks], st, ev[1], ev[2], &launches);
        if (rc) return rc;
        CASPHY_CUDA_TRY(cudaEventRecord(ev[3], st));
        std::vector<u32> eLenH(ntip), raw((size_t)2 * nedge);
        int errs[2] = {0, 0};
        CASPHY_CUDA_TRY(cudaMemcpyAsync(eLenH.data(), L.eLen, sizeof(u32) * ntip, cudaMemcpyDeviceToHost, st));
        CASPHY_CUDA_TRY(cudaMemcpyAsync(raw.data(), L.rawEdge, sizeof(u32) * 2 * nedge, cudaMemcpyDeviceToHost, st));
        CASPHY_CUDA_TRY(cudaMemcpyAsync(hst, L.stats, sizeof(hst), cudaMemcpyDeviceToHost, st));
        unsigned long long prof[joinx::PROF_N] = {0};
        if (getenv("CASPHY_PROFILE"))
            CASPHY_CUDA_TRY(cudaMemcpyAsync(prof, L.stats + 8, sizeof(prof), cudaMemcpyDeviceToHost, st));
        CASPHY_CUDA_TRY(cudaMemcpyAsync(&errs[0], L.prepErr, sizeof(int), cudaMemcpyDeviceToHost, st));
        CASPHY_CUDA_TRY(cudaMemcpyAsync(&errs[1], L.jerr, sizeof(int), cudaMemcpyDeviceToHost, st));
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
        joinx::preorder_relabel(ntip, raw.data(), edge_out, order.data());
        if (getenv("CASPHY_PROFILE")) {
            static const char* names[joinx::PROF_N] = {"barrier", "table", "decide", "build", "scan", "post",
                                                       "stale_post", "compact", "select", "stale_scan",
                                                       "sc_copy", "sc_acc", "sc_red"};
            fprintf(stderr, "join-loop sections (CTA 0, ms):");
            for (int i = 0; i < joinx::PROF_N; i++) fprintf(stderr, " %s=%.1f", names[i], prof[i] / 1e6);
            fprintf(stderr, "\n");
        }
        for (u32 i = 0; i + 1 < ntip; i++) lst.alg_bytes_init += 2ull * eLenH[i] * (u64)(ntip - 1 - i);
    } else {
        // one cell: no joins; the root row is the cell itself
        PrepArgs pa{ntip, ncol, (ncol + 7u) & ~7u, nState, 8, codes, L.Wsel, 0xFFFFu, L.nodeRow, L.eSC, L.eW,
                    L.eLen, L.prepErr};
        CASPHY_CUDA_TRY(cudaMemsetAsync(L.prepErr, 0, sizeof(int), st));
        k_prep_rows<<<1, 256, 0, st>>>(pa);
        launches = 1;
        CASPHY_CUDA_TRY(cudaEventRecord(ev[1], st));
        CASPHY_CUDA_TRY(cudaEventRecord(ev[2], st));
        CASPHY_CUDA_TRY(cudaEventRecord(ev[3], st));
    }
    CASPHY_CUDA_TRY(cudaMemcpyAsync(dOrder, order.data(), sizeof(u32) * nrows, cudaMemcpyHostToDevice, st));
    u32* sout = d_state_out ? d_state_out : dState;
    k_gather<<<nrows, 256, 0, st>>>(L.nodeRow, ncol, (ncol + 7u) & ~7u, dOrder, nrows, sout);
    launches++;
    if (h_state_out)
        CASPHY_CUDA_TRY(cudaMemcpyAsync(h_state_out, sout, sizeof(u32) * (size_t)nrows * ncol, cudaMemcpyDeviceToHost,
                                        st));
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
    lst.kernel_launches = (u64)launches;
    lst.init_scan_ms = t12;
    lst.join_loop_ms = t23;
    lst.total_ms = t04;
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
// The scratch region is the file-scope array below.  The CUDA runtime
// reserves it on a device when it loads this file's device code there: at
// context creation when modules load eagerly (CUDA_MODULE_LOADING=EAGER),
// otherwise at the first use of any kernel or symbol of this file on that
// device (the first indel join, with or without allocation).  From then on
// the GPU holds it (kScratchBytes) until the process exits.  A caller that
// hands the rest of the GPU's memory to its own pool should make its first
// call (or set CUDA_MODULE_LOADING=EAGER) before it does.  All calls on
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

// Pre-order relabelling on the device (the same walk as preorder_relabel).
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

struct Extra {
    double* w64; u16* wint; u32* wflags; u32* relabel; u32* stack; unsigned char* cursor; u32* order; u32* dfsErr;
};

static Extra carve_extra(Carve& c, u32 ntip, u32 ncol, u32 nState) {
    const u32 nnode = 2 * ntip - 1;
    const size_t nw = (size_t)nState * ncol;
    Extra e;
    e.w64 = c.take<double>(nw ? nw : 1);
    e.wint = c.take<u16>(nw ? nw : 1);
    e.wflags = c.take<u32>(4);
    e.relabel = c.take<u32>(nnode);
    e.stack = c.take<u32>(nnode);
    e.cursor = c.take<unsigned char>(nnode);
    e.order = c.take<u32>(ntip);
    e.dfsErr = c.take<u32>(1);
    return e;
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
    const u32 nChunks = (ntip + kCap - 1) / kCap;
    Carve need;
    carve_indel(need, ntip, ncol, nState, (u32)nSM, nChunks, false);
    carve_extra(need, ntip, ncol, nState);
    const size_t bytes = need.off + 256;
    if (bytes > kScratchBytes || nChunks > 64) {
        char msg[200];
        snprintf(msg, sizeof(msg),
                 "casphy_join_indel_noalloc: %u cells x %u sites need %zu bytes of scratch, the fixed limit is %zu",
                 ntip, ncol, bytes, kScratchBytes);
        casphy_set_last_error_msg(msg);
        return CASPHY_ERANGE;
    }
    void* base = nullptr;
    int rc = scratch_address(dev, &base);
    if (rc) return rc;
    std::lock_guard<std::mutex> devLock(g_dev_mu[dev & 63]);
    cudaStream_t st = (cudaStream_t)stream;
    // On every return from here on, wait for this call's work on the stream
    // before the device lock is released (destroyed before devLock), so an
    // early error return never leaves kernels using the shared scratch while
    // the next call starts to overwrite it.
    struct DrainOnReturn {
        cudaStream_t s;
        ~DrainOnReturn() { (void)cudaStreamSynchronize(s); }
    } drain{st};
    Carve c;
    c.base = static_cast<char*>(base);
    const IndelBuffers L = carve_indel(c, ntip, ncol, nState, (u32)nSM, nChunks, false);
    const Extra X = carve_extra(c, ntip, ncol, nState);
    const size_t nw = (size_t)nState * ncol;

    // weights: host float64 -> scratch, converted on the device
    if (nw) CASPHY_CUDA_TRY(cudaMemcpyAsync(X.w64, weight, sizeof(double) * nw, cudaMemcpyHostToDevice, st));
    CASPHY_CUDA_TRY(cudaMemcpyAsync(L.tipSize, tipSize, sizeof(u32) * ntip, cudaMemcpyHostToDevice, st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(X.wflags, 0, sizeof(u32) * 4, st));
    if (nw) k_weights<<<ncol, 32, 0, st>>>(X.w64, nState, ncol, L.Wsel, X.wint, X.wflags);
    u32 wf[4] = {0, 0, 0, 0};
    CASPHY_CUDA_TRY(cudaMemcpyAsync(wf, X.wflags, sizeof(wf), cudaMemcpyDeviceToHost, st));
    CASPHY_CUDA_TRY(cudaStreamSynchronize(st));
    if (wf[2]) {
        casphy_set_last_error_msg("weights must be >= 0 and not NaN");
        return CASPHY_EINVAL;
    }
    const bool intPath = !wf[0] && wf[3] <= 2048u && (u64)nState + 1 <= 0x7FFFu;
    const bool unitW = intPath && !wf[1];
    if (intPath && nw) CASPHY_CUDA_TRY(cudaMemcpyAsync(L.Wsel, X.wint, sizeof(u16) * nw, cudaMemcpyDeviceToDevice, st));
    u64 chunkStart[65];
    chunk_table(ntip, nChunks, chunkStart);
    CASPHY_CUDA_TRY(cudaMemcpyAsync(L.chunkStart, chunkStart, sizeof(u64) * (nChunks + 1), cudaMemcpyHostToDevice,
                                    st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(X.dfsErr, 0, sizeof(u32), st));
    int launches = 0;
    rc = launch_indel(L, ntip, ncol, nState, d_codes, intPath, unitW, false, minSize, minRatio, (u32)nSM, nChunks,
                      chunkStart[nChunks], st, nullptr, nullptr, &launches);
    if (rc) return rc;
    k_preorder<<<1, 32, 0, st>>>(L.rawEdge, ntip, X.relabel, X.stack, X.cursor, d_edge_out, X.order, X.dfsErr);
    k_gather<<<ntip - 1, 256, 0, st>>>(L.nodeRow, ncol, (ncol + 7u) & ~7u, X.order, ntip - 1, d_state_out);
    CASPHY_CUDA_TRY(cudaGetLastError());
    int errs[2] = {0, 0};
    u32 dfsErr = 0;
    CASPHY_CUDA_TRY(cudaMemcpyAsync(&errs[0], L.prepErr, sizeof(int), cudaMemcpyDeviceToHost, st));
    CASPHY_CUDA_TRY(cudaMemcpyAsync(&errs[1], L.jerr, sizeof(int), cudaMemcpyDeviceToHost, st));
    CASPHY_CUDA_TRY(cudaMemcpyAsync(&dfsErr, X.dfsErr, sizeof(u32), cudaMemcpyDeviceToHost, st));
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
