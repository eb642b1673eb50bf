// Bit-join model for the persistent join engine (cu/joinEdgeBitReverse.cu):
// query entries, the three exact scoring paths, node states, and the per-tip
// preparation and initial-scan tile shared by the single-join launch and the
// batched bootstrap.
#pragma once
#include "join_engine.cuh"

namespace casphy {
namespace bitjoin {

using joinx::kNone;
using joinx::kThreads;
constexpr u32 kG = 4;                  // candidates per thread
constexpr u32 kCap = kThreads * kG;    // 2048 candidates per pass
constexpr u32 kMaxBin = 4096;          // 131072 sites
enum { PATH_UNIT = 0, PATH_PLANES = 1, PATH_FLOAT = 2 };

// E entry: word | plane << 16, and the (plane-masked) query word.
struct QueryArgs {
    u32 nbin, nplanes;
    const u32* planeMask;  // nplanes x nbin
};

// Appends the query entries of one row (ascending words, planes inside a
// word) into eW/eQ; one CTA.  Returns the count.
__device__ inline int build_bit_entries(const QueryArgs& q, const u32* rowSmem, u32* eW, u32* eQ, u32* wcount) {
    const u32 lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const u32 P = q.nplanes ? q.nplanes : 1;
    int base = 0;
    for (u32 w0 = 0; w0 < q.nbin; w0 += kThreads) {
        const u32 w = w0 + threadIdx.x;
        u32 cnt = 0;
        const u32 qw = w < q.nbin ? rowSmem[w] : 0u;
        if (qw) {
            if (!q.nplanes) cnt = 1;
            else
                for (u32 k = 0; k < P; k++) cnt += (qw & q.planeMask[(size_t)k * q.nbin + w]) != 0u;
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
        u32 pos = base + wcount[16 + wid] + incl - cnt;
        if (qw) {
            if (!q.nplanes) {
                eW[pos] = w;
                eQ[pos] = qw;
            } else {
                for (u32 k = 0; k < P; k++) {
                    const u32 m = qw & q.planeMask[(size_t)k * q.nbin + w];
                    if (m) {
                        eW[pos] = w | (k << 16);
                        eQ[pos] = m;
                        pos++;
                    }
                }
            }
        }
        base += (int)wcount[32];
        __syncthreads();
    }
    return base;
}

template <int PATH>
__device__ __forceinline__ void score4(const u32* __restrict__ col, u32 Sp, u32 cb, const u32* eW, const u32* eQ,
                                       int e0, int nE, int step, const float* __restrict__ wf, u32 acc[4],
                                       float facc[4]) {
    if (PATH == PATH_FLOAT) {
        for (int e = e0; e < nE; e += step) {
            const u32 w = eW[e], q = eQ[e];
            const uint4 v = ld_cg_v4(col + (size_t)w * Sp + cb);
            const u32 x[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int i = 0; i < 4; i++) {
                u32 m = q & x[i];
                while (m) {
                    const int bit = __ffs(m) - 1;
                    facc[i] += __ldg(wf + w * 32 + bit);
                    m &= m - 1;
                }
            }
        }
        return;
    }
    int e = e0;
    for (; e + 3 * step < nE; e += 4 * step) {
        u32 ew[4], eq[4];
        uint4 v[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            ew[j] = eW[e + j * step];
            eq[j] = eQ[e + j * step];
        }
#pragma unroll
        for (int j = 0; j < 4; j++) v[j] = ld_cg_v4(col + (size_t)(ew[j] & 0xFFFFu) * Sp + cb);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const u32 sh = ew[j] >> 16;
            acc[0] += (u32)__popc(eq[j] & v[j].x) << sh;
            acc[1] += (u32)__popc(eq[j] & v[j].y) << sh;
            acc[2] += (u32)__popc(eq[j] & v[j].z) << sh;
            acc[3] += (u32)__popc(eq[j] & v[j].w) << sh;
        }
    }
    for (; e < nE; e += step) {
        const u32 ew = eW[e], eq = eQ[e], sh = ew >> 16;
        const uint4 v = ld_cg_v4(col + (size_t)(ew & 0xFFFFu) * Sp + cb);
        acc[0] += (u32)__popc(eq & v.x) << sh;
        acc[1] += (u32)__popc(eq & v.y) << sh;
        acc[2] += (u32)__popc(eq & v.z) << sh;
        acc[3] += (u32)__popc(eq & v.w) << sh;
    }
}

template <int PATH>
struct BitModel {
    static constexpr bool kFusedStale = false;  // stale batches rescan one query at a time
    struct Args {
        u32 nbin, nbinP, nplanes;
        int ancType;
        const u32* planeMask;
        const float* wf;
        u32* nodeSeq;
        u32* nodeBis;
        u32* colT[2];
    };
    struct Smem {
        u32* part;  // kCap u32 (per-group partial sums)
        u32* eW;
        u32* eQ;
        u32* mseq;
        u32* mbis;
    };
    __host__ __device__ static size_t engine_smem_bytes(u32 nCTA, u32 Rmax, u32 deathWords = 0, u32 pre = 0) {
        return joinx::engine_smem(nCTA, Rmax, deathWords, pre);
    }
    __host__ static size_t model_smem_bytes(const Args& m) {
        const size_t ne = (size_t)m.nbin * (m.nplanes ? m.nplanes : 1);
        return sizeof(u32) * (kCap + 2 * ne + 2 * m.nbinP) + 16;
    }
    __device__ static void carve_smem(const Args& m, unsigned char* p, Smem& s) {
        const size_t ne = (size_t)m.nbin * (m.nplanes ? m.nplanes : 1);
        s.part = reinterpret_cast<u32*>(p);
        s.eW = s.part + kCap;
        s.eQ = s.eW + ne;
        s.mseq = s.eQ + ne;
        s.mbis = s.mseq + m.nbinP;
    }
    __device__ static u32* col(const Args& m, u32 buf) { return buf ? m.colT[1] : m.colT[0]; }
    __device__ static int build_stale(const Args& m, Smem& s, u32 j1, u32* wc) {
        const u32* src = m.nodeSeq + (size_t)j1 * m.nbinP;
        for (u32 w = threadIdx.x; w < m.nbinP; w += kThreads) s.mseq[w] = w < m.nbin ? ld_cg_u32(src + w) : 0u;
        __syncthreads();
        QueryArgs q{m.nbin, PATH == PATH_PLANES ? m.nplanes : 0u, m.planeMask};
        return build_bit_entries(q, s.mseq, s.eW, s.eQ, wc);
    }
    // ancestral rules (updateAncestralKernel / updateAncestralKernel2,
    // cu/joinEdgeBitReverse.cu:77-113)
    __device__ static int build_join(const Args& m, Smem& s, u32 j1, u32 j2, u32, u32, u32* wc) {
        const u32* a1 = m.nodeSeq + (size_t)j1 * m.nbinP;
        const u32* b1 = m.nodeBis + (size_t)j1 * m.nbinP;
        const u32* a2 = m.nodeSeq + (size_t)j2 * m.nbinP;
        const u32* b2 = m.nodeBis + (size_t)j2 * m.nbinP;
        for (u32 w = threadIdx.x; w < m.nbinP; w += kThreads) {
            u32 sq = 0, bs = 0;
            if (w < m.nbin) {
                const u32 s1 = ld_cg_u32(a1 + w), s2 = ld_cg_u32(a2 + w);
                const u32 bs1 = ld_cg_u32(b1 + w), bs2 = ld_cg_u32(b2 + w);
                if (m.ancType == 0) {
                    const u32 diff = s1 ^ s2;
                    const u32 conflict = diff & (bs1 | bs2);
                    sq = (s1 | s2) & ~conflict;
                    bs = (diff & ~(bs1 ^ bs2)) | (bs1 & bs2);
                } else {
                    sq = (s1 & s2) | (bs1 & s2) | (bs2 & s1);
                    bs = (s1 ^ s2) & ~(bs1 | bs2);
                }
            }
            s.mseq[w] = sq;
            s.mbis[w] = bs;
        }
        __syncthreads();
        QueryArgs q{m.nbin, PATH == PATH_PLANES ? m.nplanes : 0u, m.planeMask};
        return build_bit_entries(q, s.mseq, s.eW, s.eQ, wc);
    }
    // slice `part` of `nparts` of the new node's rows (the engine writes them whole)
    __device__ static void store_node(const Args& m, Smem& s, u32 newNode, u32 part, u32 nparts) {
        u32* ds = m.nodeSeq + (size_t)newNode * m.nbinP;
        u32* db = m.nodeBis + (size_t)newNode * m.nbinP;
        const u32 per = (m.nbinP + nparts - 1) / nparts, w1 = min(m.nbinP, (part + 1) * per);
        for (u32 w = part * per + threadIdx.x; w < w1; w += kThreads) {
            ds[w] = s.mseq[w];
            db[w] = s.mbis[w];
        }
    }
    // slice `part` of `nparts` of slot c1's column (the engine gives the whole
    // column to c1's owner)
    __device__ static void store_slot(const Args& m, Smem& s, u32 buf, const joinx::Range& rg, u32 c1, u32 part,
                                      u32 nparts) {
        u32* c = col(m, buf);
        const u32 per = (m.nbin + nparts - 1) / nparts, w1 = min(m.nbin, (part + 1) * per);
        for (u32 w = part * per + threadIdx.x; w < w1; w += kThreads) c[(size_t)w * rg.Sp + c1] = s.mseq[w];
    }
    __device__ static u32 pass_cap(const Args&, u32 R) {
        u32 F = 1;
        if (PATH != PATH_FLOAT) {
            while (F < 16 && (u32)(kCap / (F * 2)) >= R) F *= 2;
        }
        return kCap / F;
    }
    __device__ static void score_pass(const Args& m, Smem& s, u32 buf, const joinx::Range& rg, u32 base, u32 cap,
                                      int nE, u32* ordOut) {
        const u32 F = kCap / cap, Tg = kThreads / F;
        const u32 g = threadIdx.x / Tg, t = threadIdx.x % Tg;
        const u32 cb = base + t * kG;
        u32 acc[4] = {0, 0, 0, 0};
        float facc[4] = {0.f, 0.f, 0.f, 0.f};
        if (cb < rg.hi) score4<PATH>(col(m, buf), rg.Sp, cb, s.eW, s.eQ, (int)g, nE, (int)F, m.wf, acc, facc);
        if (PATH == PATH_FLOAT) {
            *reinterpret_cast<uint4*>(s.part + t * kG) =
                make_uint4(__float_as_uint(facc[0]), __float_as_uint(facc[1]), __float_as_uint(facc[2]),
                           __float_as_uint(facc[3]));
        } else {
            *reinterpret_cast<uint4*>(s.part + g * cap + t * kG) = make_uint4(acc[0], acc[1], acc[2], acc[3]);
        }
        __syncthreads();
        for (u32 x = threadIdx.x; x < cap && base + x < rg.hi; x += kThreads) {
            float v;
            if (PATH == PATH_FLOAT) {
                v = __uint_as_float(s.part[x]);
            } else {
                u32 sum = 0;
                for (u32 gg = 0; gg < F; gg++) sum += s.part[gg * cap + x];
                v = (float)sum;
            }
            ordOut[x] = ord_f32(v);
        }
        __syncthreads();
    }
    __device__ static void compact_prepare(const Args&, Smem&, u32, const joinx::Range&) {}
    __device__ static void compact_move(const Args& m, Smem&, u32 buf, u32 nb, const joinx::Range& rg, u32 Spn,
                                        const u32* ranks, const u32*) {
        const u32* src = col(m, buf);
        u32* dst = col(m, nb);
        const u32 R = rg.hi - rg.lo;
        for (u32 w = 0; w < m.nbin; w++) {
            for (u32 x = threadIdx.x; x < R; x += kThreads) {
                const u32 r = ranks[x];
                if (r != kNone) dst[(size_t)w * Spn + r] = ld_cg_u32(src + (size_t)w * rg.Sp + rg.lo + x);
            }
        }
    }
    __device__ static void after_compact(const Args&, Smem&, u32, const joinx::Range&) {}
};

// One warp prepares tip `tip` from its row `src`: node rows (seq = input,
// bistate = 0), its column of the slot matrix and its query entries.
__device__ __forceinline__ void prep_tip(const u32* __restrict__ src, u32 tip, u32 nbin, u32 nbinP, u32 Sp,
                                         u32 nplanes, const u32* __restrict__ planeMask, u32* nodeSeq, u32* nodeBis,
                                         u32* colT, u32* eW, u32* eQ, u32* eLen, u32 eStride) {
    const u32 lane = threadIdx.x & 31;
    u32 n = 0;
    const u32 P = nplanes ? nplanes : 1;
    for (u32 w0 = 0; w0 < nbinP; w0 += 32) {
        const u32 w = w0 + lane;
        const u32 v = w < nbin ? src[w] : 0u;
        if (w < nbinP) {
            nodeSeq[(size_t)tip * nbinP + w] = v;
            nodeBis[(size_t)tip * nbinP + w] = 0u;
        }
        if (w < nbin) colT[(size_t)w * Sp + tip] = v;
        for (u32 k = 0; k < P; k++) {
            const u32 m = nplanes ? (v & (w < nbin ? planeMask[(size_t)k * nbin + w] : 0u)) : v;
            const u32 bal = __ballot_sync(0xFFFFFFFFu, m != 0u);
            if (m) {
                const u32 pos = n + __popc(bal & ((1u << lane) - 1u));
                eW[(size_t)tip * eStride + pos] = w | (k << 16);
                eQ[(size_t)tip * eStride + pos] = m;
            }
            n += __popc(bal);
        }
    }
    if (lane == 0) eLen[tip] = n;
}

// Entries of one tip are ordered by plane inside each 32-word block; the
// integer paths do not depend on order and the float path uses one plane, so
// the ascending-bit order of the reference is kept where it matters.

struct InitArgs {
    u32 ntip, nbin, Sp, eStride;
    const u32* colT;
    const u32* eW;
    const u32* eQ;
    const u32* eLen;
    const float* wf;
    const u64* chunkStart;
    u32 nChunks;
    u64 nTiles;
    unsigned long long* tileCounter;
    unsigned long long* initKey;
};

// Initial-scan tile t: query q against the candidates of one 2048-slot chunk
// above it; the best (value, smaller node) key goes to initKey[q].
template <int PATH>
__device__ __forceinline__ void init_tile(const InitArgs& a, u64 t, u64* red) {
    u32 k = 0;
    while (k + 1 < a.nChunks && a.chunkStart[k + 1] <= t) k++;
    const u32 q = (u32)(t - a.chunkStart[k]);
    const u32 cb = k * kCap + threadIdx.x * kG;
    u64 best = make_key(ORD_F32_NEG1, 0u);
    if (cb < a.ntip && cb + kG > q + 1) {
        u32 acc[4] = {0, 0, 0, 0};
        float facc[4] = {0.f, 0.f, 0.f, 0.f};
        score4<PATH>(a.colT, a.Sp, cb, a.eW + (size_t)q * a.eStride, a.eQ + (size_t)q * a.eStride, 0,
                     (int)a.eLen[q], 1, a.wf, acc, facc);
#pragma unroll
        for (u32 i = 0; i < kG; i++) {
            const u32 j = cb + i;
            if (j > q && j < a.ntip) {
                const float v = PATH == PATH_FLOAT ? facc[i] : (float)acc[i];
                const u64 key = make_key(ord_f32(v), j);
                best = key > best ? key : best;
            }
        }
    }
    best = block_max_u64(best, red);
    if (threadIdx.x == 0) atomicMax(a.initKey + q, (unsigned long long)best);
}

}  // namespace bitjoin
}  // namespace casphy
