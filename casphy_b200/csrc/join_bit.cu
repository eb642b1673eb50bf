// Greedy join of bit-coded cells on B200 (replaces cu/joinEdgeBitReverse.cu).
//
// score(q, c) = sum over the query's set bits b that are also set in c of
// w[b], added in binary32 in ascending bit order (cu/joinEdgeBitReverse.cu:
// 53-75 with the bit list of calculateSharedPacked :233-244).  Three exact
// evaluations:
//  * UNIT  (every w = 1): popcount(q & c) per word.
//  * PLANES (every w a non-negative integer, total <= 2^24, so every binary32
//    partial sum is exact): w is split into bit planes; plane k masks the
//    sites whose weight has bit k, score = sum_k 2^k popcount(q & mask_k & c).
//  * FLOAT (anything else): per candidate, the matching bits are visited in
//    ascending order and added in binary32, as the reference does.
// Node state is the (seq, bistate) pair of cu/joinEdgeBitReverse.cu:77-113;
// rows are output as seq & ~bistate (:115-121).  Candidate rows live
// column-major by slot (word w of slots c..c+3 is one 16-byte load).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "join_engine.cuh"
#include "runtime.h"

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
__device__ int build_bit_entries(const QueryArgs& q, const u32* rowSmem, u32* eW, u32* eQ, u32* wcount) {
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
    __host__ __device__ static size_t engine_smem_bytes(u32 nCTA, u32 Rmax) { return joinx::engine_smem(nCTA, Rmax); }
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
    __device__ static void store_node(const Args& m, Smem& s, u32 newNode) {
        u32* ds = m.nodeSeq + (size_t)newNode * m.nbinP;
        u32* db = m.nodeBis + (size_t)newNode * m.nbinP;
        for (u32 w = threadIdx.x; w < m.nbinP; w += kThreads) {
            ds[w] = s.mseq[w];
            db[w] = s.mbis[w];
        }
    }
    __device__ static void store_slot(const Args& m, Smem& s, u32 buf, const joinx::Range& rg, u32 c1, u32) {
        u32* c = col(m, buf);
        for (u32 w = threadIdx.x; w < m.nbin; w += kThreads) c[(size_t)w * rg.Sp + c1] = s.mseq[w];
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

// --- preparation and initial scan ------------------------------------------

// One warp per tip: node rows (seq = input, bistate = 0), the column-major
// slot matrix, and the tip's query entries.
__global__ void k_prep(const u32* __restrict__ words, u32 ntip, u32 nbin, u32 nbinP, u32 Sp, u32 nplanes,
                       const u32* __restrict__ planeMask, u32* nodeSeq, u32* nodeBis, u32* colT, u32* eW, u32* eQ,
                       u32* eLen, u32 eStride) {
    const u32 warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const u32 lane = threadIdx.x & 31;
    if (warp >= ntip) return;
    const u32* src = words + (size_t)warp * nbin;
    u32 n = 0;
    const u32 P = nplanes ? nplanes : 1;
    for (u32 w0 = 0; w0 < nbinP; w0 += 32) {
        const u32 w = w0 + lane;
        const u32 v = w < nbin ? src[w] : 0u;
        if (w < nbinP) {
            nodeSeq[(size_t)warp * nbinP + w] = v;
            nodeBis[(size_t)warp * nbinP + w] = 0u;
        }
        if (w < nbin) colT[(size_t)w * Sp + warp] = v;
        for (u32 k = 0; k < P; k++) {
            const u32 m = nplanes ? (v & (w < nbin ? planeMask[(size_t)k * nbin + w] : 0u)) : v;
            const u32 bal = __ballot_sync(0xFFFFFFFFu, m != 0u);
            if (m) {
                const u32 pos = n + __popc(bal & ((1u << lane) - 1u));
                eW[(size_t)warp * eStride + pos] = w | (k << 16);
                eQ[(size_t)warp * eStride + pos] = m;
            }
            n += __popc(bal);
        }
    }
    if (lane == 0) eLen[warp] = n;
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

template <int PATH>
__global__ void __launch_bounds__(kThreads) k_init(InitArgs a) {
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
        cur ^= 1;
        __syncthreads();
    }
}

__global__ void k_gather_bit(const u32* __restrict__ nodeSeq, const u32* __restrict__ nodeBis, u32 nbin, u32 nbinP,
                             const u32* __restrict__ order, u32 nrows, u32* __restrict__ out) {
    const u32 r = blockIdx.x;
    if (r >= nrows) return;
    const size_t o = (size_t)order[r] * nbinP;
    for (u32 w = threadIdx.x; w < nbin; w += blockDim.x) out[(size_t)r * nbin + w] = nodeSeq[o + w] & ~nodeBis[o + w];
}

}  // namespace bitjoin

using namespace bitjoin;

template <int PATH>
static int launch_bit_join(joinx::Common& c, typename BitModel<PATH>::Args m, u32 nCTA, cudaStream_t st) {
    using M = BitModel<PATH>;
    const size_t smem = M::engine_smem_bytes(nCTA, c.Rmax) + M::model_smem_bytes(m);
    void* fn = (void*)joinx::k_join<M>;
    CASPHY_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int perSM = 0;
    CASPHY_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, fn, kThreads, smem));
    if (perSM < 1) {
        casphy_set_last_error_msg("bit join kernel does not fit on an SM (too many words)");
        return CASPHY_ERANGE;
    }
    void* args[] = {&c, &m};
    CASPHY_CUDA_TRY(cudaLaunchCooperativeKernel(fn, dim3(nCTA), dim3(kThreads), args, smem, st));
    return CASPHY_OK;
}

template <int PATH>
static int launch_bit_init(const InitArgs& ia, u32 nSM, cudaStream_t st) {
    int perSM = 0;
    CASPHY_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_init<PATH>, kThreads, 0));
    k_init<PATH><<<nSM * std::max(perSM, 1), kThreads, 0, st>>>(ia);
    return CASPHY_OK;
}

static int join_bit_impl(u32 ntip, u32 nbin, const u32* d_words, const u32* h_words, const double* weight,
                         int ancType, u32* edge_out, u32* d_state_out, u32* h_state_out, casphy_join_stats* stats,
                         cudaStream_t st) {
    if (ntip == 0 || nbin == 0 || !weight || !edge_out) return CASPHY_EINVAL;
    if (nbin > kMaxBin) {
        casphy_set_last_error_msg("nbin exceeds 4096 words");
        return CASPHY_ERANGE;
    }
    const u32 nsite = nbin * 32;
    std::vector<float> wf(nsite);
    bool unit = true, integral = true;
    double total = 0;
    u32 maxw = 0;
    for (u32 i = 0; i < nsite; i++) {
        const double x = weight[i];
        if (std::isnan(x) || x < 0) {
            casphy_set_last_error_msg("weights must be >= 0 and not NaN");
            return CASPHY_EINVAL;
        }
        wf[i] = (float)x;
        if (wf[i] != 1.0f) unit = false;
        if (!(wf[i] == std::floor(wf[i]) && wf[i] < 16777216.0f)) integral = false;
        total += wf[i];
        if (integral) maxw = std::max(maxw, (u32)wf[i]);
    }
    if (total > 16777216.0) integral = false;
    const int path = unit ? PATH_UNIT : (integral ? PATH_PLANES : PATH_FLOAT);
    u32 nplanes = 0;
    std::vector<u32> planes;
    if (path == PATH_PLANES) {
        while ((1u << nplanes) <= maxw && nplanes < 24) nplanes++;
        if (nplanes == 0) nplanes = 1;
        planes.assign((size_t)nplanes * nbin, 0u);
        for (u32 i = 0; i < nsite; i++) {
            const u32 v = (u32)wf[i];
            for (u32 k = 0; k < nplanes; k++)
                if ((v >> k) & 1u) planes[(size_t)k * nbin + i / 32] |= 1u << (i % 32);
        }
    }
    const u32 P = nplanes ? nplanes : 1;
    casphy_join_stats lst{};
    lst.int_path = path == PATH_FLOAT ? 0 : 1;
    DeviceScope ds;
    int nSM = 0;
    CASPHY_CUDA_TRY(cudaDeviceGetAttribute(&nSM, cudaDevAttrMultiProcessorCount, ds.dev));
    const u32 nCTA = (u32)nSM;
    const u32 nnode = 2 * ntip - 1, nedge = 2 * ntip - 2, nrows = std::max(ntip - 1, 1u);
    const u32 nbinP = (nbin + 3u) & ~3u, Sp = (ntip + 7u) & ~7u;
    const u32 eStride = nbin * P;
    const u32 nChunks = (ntip + kCap - 1) / kCap;
    auto carve = [&](Carve& c) {
        struct B {
            u32* words; u32* planeMask; float* wf; u32* nodeSeq; u32* nodeBis; u32* colT0; u32* colT1; u32* lm[6];
            u32* node2slot; u32* nodeDeath; u32* nodeSize; u32* rawEdge; u32* eW; u32* eQ; u32* eLen;
            unsigned long long* initKey; joinx::BlockRec* pub; u32* pubCnt; u64* partial; u32* counts; u32* flags;
            int* jerr; unsigned long long* tileCounter; u64* chunkStart; unsigned long long* stats; u32* tip;
            u32* order; u32* state;
        } b;
        b.words = c.take<u32>(h_words ? (size_t)ntip * nbin : 0);
        b.planeMask = c.take<u32>((size_t)P * nbin);
        b.wf = c.take<float>(nsite);
        b.nodeSeq = c.take<u32>((size_t)nnode * nbinP);
        b.nodeBis = c.take<u32>((size_t)nnode * nbinP);
        b.colT0 = c.take<u32>((size_t)nbin * Sp);
        b.colT1 = c.take<u32>((size_t)nbin * Sp);
        for (int i = 0; i < 6; i++) b.lm[i] = c.take<u32>(Sp);
        b.node2slot = c.take<u32>(nnode);
        b.nodeDeath = c.take<u32>(nnode);
        b.nodeSize = c.take<u32>(nnode);
        b.rawEdge = c.take<u32>((size_t)2 * nedge + 2);
        b.eW = c.take<u32>((size_t)ntip * eStride);
        b.eQ = c.take<u32>((size_t)ntip * eStride);
        b.eLen = c.take<u32>(ntip);
        b.initKey = c.take<unsigned long long>(ntip);
        b.pub = c.take<joinx::BlockRec>(4 * nCTA);
        b.pubCnt = c.take<u32>(2 * nCTA);
        b.partial = c.take<u64>(2 * nCTA);
        b.counts = c.take<u32>(nCTA);
        b.flags = c.take<u32>(16 * nCTA);
        b.jerr = c.take<int>(1);
        b.tileCounter = c.take<unsigned long long>(1);
        b.chunkStart = c.take<u64>(nChunks + 1);
        b.stats = c.take<unsigned long long>(8);
        b.tip = c.take<u32>(ntip);
        b.order = c.take<u32>(nrows);
        b.state = c.take<u32>(h_state_out ? (size_t)nrows * nbin : 0);
        return b;
    };
    Carve cv;
    carve(cv);
    void* base = nullptr;
    int rc = ds.reserve(cv.off + 256, &base);
    if (rc) return rc;
    Carve c2;
    c2.base = static_cast<char*>(base);
    const auto L = carve(c2);
    cudaEvent_t ev[5];
    for (auto& e : ev) CASPHY_CUDA_TRY(cudaEventCreate(&e));
    CASPHY_CUDA_TRY(cudaEventRecord(ev[0], st));
    const u32* words = d_words;
    if (h_words) {
        CASPHY_CUDA_TRY(cudaMemcpyAsync(L.words, h_words, sizeof(u32) * (size_t)ntip * nbin, cudaMemcpyHostToDevice, st));
        words = L.words;
    }
    if (nplanes)
        CASPHY_CUDA_TRY(cudaMemcpyAsync(L.planeMask, planes.data(), sizeof(u32) * planes.size(), cudaMemcpyHostToDevice,
                                        st));
    CASPHY_CUDA_TRY(cudaMemcpyAsync(L.wf, wf.data(), sizeof(float) * nsite, cudaMemcpyHostToDevice, st));
    std::vector<u32> ones(ntip, 1u);
    CASPHY_CUDA_TRY(cudaMemcpyAsync(L.tip, ones.data(), sizeof(u32) * ntip, cudaMemcpyHostToDevice, st));
    std::vector<u64> chunkStart(nChunks + 1, 0);
    for (u32 k = 0; k < nChunks; k++) {
        const u64 end = std::min<u64>((u64)(k + 1) * kCap, ntip);
        chunkStart[k + 1] = chunkStart[k] + (end >= 1 ? end - 1 : 0);
    }
    CASPHY_CUDA_TRY(cudaMemcpyAsync(L.chunkStart, chunkStart.data(), sizeof(u64) * (nChunks + 1),
                                    cudaMemcpyHostToDevice, st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(L.jerr, 0, sizeof(int), st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(L.flags, 0, sizeof(u32) * 16 * nCTA, st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(L.tileCounter, 0, sizeof(unsigned long long), st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(L.stats, 0, sizeof(unsigned long long) * 8, st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(L.colT0, 0, sizeof(u32) * (size_t)nbin * Sp, st));
    k_prep<<<(ntip + 7) / 8, 256, 0, st>>>(words, ntip, nbin, nbinP, Sp, nplanes, L.planeMask, L.nodeSeq, L.nodeBis,
                                           L.colT0, L.eW, L.eQ, L.eLen, eStride);
    joinx::k_fill_u64<<<(ntip + 255) / 256, 256, 0, st>>>(L.initKey, ntip, ((u64)ORD_F32_NEG1 << 32) | 0xFFFFFFFFull);
    int launches = 2;
    std::vector<u32> order(nrows, 0u);
    unsigned long long hst[8] = {0};
    CASPHY_CUDA_TRY(cudaEventRecord(ev[1], st));
    if (ntip >= 2) {
        InitArgs ia{ntip, nbin, Sp, eStride, L.colT0, L.eW, L.eQ, L.eLen, L.wf, L.chunkStart, nChunks,
                    chunkStart[nChunks], L.tileCounter, L.initKey};
        rc = path == PATH_UNIT ? launch_bit_init<PATH_UNIT>(ia, nSM, st)
             : path == PATH_PLANES ? launch_bit_init<PATH_PLANES>(ia, nSM, st)
                                   : launch_bit_init<PATH_FLOAT>(ia, nSM, st);
        if (rc) return rc;
        launches++;
    }
    CASPHY_CUDA_TRY(cudaEventRecord(ev[2], st));
    if (ntip >= 2) {
        joinx::k_slot_init<<<(std::max(Sp, nnode) + 255) / 256, 256, 0, st>>>(
            ntip, Sp, nnode, L.initKey, ORD_F32_NEG1, L.lm[0], L.lm[1], L.lm[2], L.node2slot, L.nodeDeath, L.nodeSize,
            L.tip);
        joinx::Common c{};
        c.ntip = ntip; c.nnode = nnode; c.nCTA = nCTA; c.align = 8;
        c.lmOrd[0] = L.lm[0]; c.lmIdx[0] = L.lm[1]; c.slotNode[0] = L.lm[2];
        c.lmOrd[1] = L.lm[3]; c.lmIdx[1] = L.lm[4]; c.slotNode[1] = L.lm[5];
        c.node2slot = L.node2slot; c.nodeDeath = L.nodeDeath; c.nodeSize = L.nodeSize; c.rawEdge = L.rawEdge;
        c.pub = L.pub; c.pubCnt = L.pubCnt; c.partial = L.partial; c.counts = L.counts; c.flags = L.flags;
        c.err = L.jerr; c.limitNs = 20ull * 1000 * 1000 * 1000; c.statsOut = L.stats;
        c.Rmax = (((ntip + nCTA - 1) / nCTA) + 7u) & ~7u;
        c.ordNeg1 = ORD_F32_NEG1; c.compactMin = 4096; c.compactQ8 = 192; c.bytesPerPairSite = 4000;
        if (path == PATH_UNIT) {
            BitModel<PATH_UNIT>::Args m{nbin, nbinP, 0, ancType, L.planeMask, L.wf, L.nodeSeq, L.nodeBis,
                                        {L.colT0, L.colT1}};
            rc = launch_bit_join<PATH_UNIT>(c, m, nCTA, st);
        } else if (path == PATH_PLANES) {
            BitModel<PATH_PLANES>::Args m{nbin, nbinP, nplanes, ancType, L.planeMask, L.wf, L.nodeSeq, L.nodeBis,
                                          {L.colT0, L.colT1}};
            rc = launch_bit_join<PATH_PLANES>(c, m, nCTA, st);
        } else {
            BitModel<PATH_FLOAT>::Args m{nbin, nbinP, 0, ancType, L.planeMask, L.wf, L.nodeSeq, L.nodeBis,
                                         {L.colT0, L.colT1}};
            rc = launch_bit_join<PATH_FLOAT>(c, m, nCTA, st);
        }
        if (rc) return rc;
        launches += 2;
    }
    CASPHY_CUDA_TRY(cudaEventRecord(ev[3], st));
    if (ntip >= 2) {
        std::vector<u32> raw((size_t)2 * nedge);
        int jerr = 0;
        CASPHY_CUDA_TRY(cudaMemcpyAsync(raw.data(), L.rawEdge, sizeof(u32) * 2 * nedge, cudaMemcpyDeviceToHost, st));
        CASPHY_CUDA_TRY(cudaMemcpyAsync(hst, L.stats, sizeof(hst), cudaMemcpyDeviceToHost, st));
        CASPHY_CUDA_TRY(cudaMemcpyAsync(&jerr, L.jerr, sizeof(int), cudaMemcpyDeviceToHost, st));
        CASPHY_CUDA_TRY(cudaStreamSynchronize(st));
        if (jerr) {
            casphy_set_last_error_msg(jerr == CASPHY_ETIMEOUT ? "join loop grid barrier timed out"
                                                               : "join loop invariant violated");
            return jerr;
        }
        joinx::preorder_relabel(ntip, raw.data(), edge_out, order.data());
    }
    CASPHY_CUDA_TRY(cudaMemcpyAsync(L.order, order.data(), sizeof(u32) * nrows, cudaMemcpyHostToDevice, st));
    u32* sout = d_state_out ? d_state_out : L.state;
    k_gather_bit<<<nrows, 128, 0, st>>>(L.nodeSeq, L.nodeBis, nbin, nbinP, L.order, nrows, sout);
    launches++;
    if (h_state_out)
        CASPHY_CUDA_TRY(cudaMemcpyAsync(h_state_out, sout, sizeof(u32) * (size_t)nrows * nbin, cudaMemcpyDeviceToHost,
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

extern "C" int casphy_join_bit(uint32_t ntip, uint32_t nbin, const uint32_t* words, const double* weight,
                               int ancestralType, uint32_t* edge_out, uint32_t* state_out,
                               casphy_join_stats* stats) {
    int rc = casphy::require_device();
    if (rc) return rc;
    if (!words || !state_out) return CASPHY_EINVAL;
    return casphy::join_bit_impl(ntip, nbin, nullptr, words, weight, ancestralType ? 1 : 0, edge_out, nullptr,
                                 state_out, stats, 0);
}

extern "C" int casphy_join_bit_dev(uint32_t ntip, uint32_t nbin, const uint32_t* d_words, const double* weight,
                                   int ancestralType, uint32_t* edge_out, uint32_t* d_state_out,
                                   casphy_join_stats* stats, void* stream) {
    int rc = casphy::require_device();
    if (rc) return rc;
    if (!d_words) return CASPHY_EINVAL;
    return casphy::join_bit_impl(ntip, nbin, d_words, nullptr, weight, ancestralType ? 1 : 0, edge_out,
                                 d_state_out, nullptr, stats, (cudaStream_t)stream);
}
