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

#include "join_bit_model.cuh"
#include "runtime.h"

namespace casphy {
namespace bitjoin {

// --- preparation and initial scan ------------------------------------------

__global__ void k_prep(const u32* __restrict__ words, u32 ntip, u32 nbin, u32 nbinP, u32 Sp, u32 nplanes,
                       const u32* __restrict__ planeMask, u32* nodeSeq, u32* nodeBis, u32* colT, u32* eW, u32* eQ,
                       u32* eLen, u32 eStride) {
    const u32 warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (warp >= ntip) return;
    prep_tip(words + (size_t)warp * nbin, warp, nbin, nbinP, Sp, nplanes, planeMask, nodeSeq, nodeBis, colT, eW, eQ,
             eLen, eStride);
}

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
        init_tile<PATH>(a, t, red);
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
    // the joined-node bitmap only where shared memory allows it
    int smemMax = 0, dev = 0;
    CASPHY_CUDA_TRY(cudaGetDevice(&dev));
    CASPHY_CUDA_TRY(cudaDeviceGetAttribute(&smemMax, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    if (M::engine_smem_bytes(nCTA, c.Rmax, c.deathWords) + M::model_smem_bytes(m) > (size_t)smemMax - 4096)
        c.deathWords = 0;
    const size_t smem = M::engine_smem_bytes(nCTA, c.Rmax, c.deathWords) + M::model_smem_bytes(m);
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
        b.partial = c.take<u64>((size_t)2 * nCTA * joinx::kMaxBatch);
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
        c.maxBatch = joinx::stale_batch_setting();
        c.deathWords = (nnode + 31) / 32;
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
