// tipMerge on B200 (replaces cu/tipMerge.cu): categories of tips whose
// radius-neighbour lists overlap.
//
// The reference visits rows in chunks of 131072 candidate columns; for each
// row j it collects the later neighbours k of the chunk that pass its filter,
// launches one kernel for their shared-neighbour counts |N(j) n N(k)| and
// merges categories on the host in list order (cu/tipMerge.cu:318-426).
// The counts do not depend on the merges, so here one launch computes them
// for every (j, k > j) pair of the lists up front (one warp per pair: each
// element of the shorter list is looked up in the longer one by binary
// search), and the host replays the reference's visiting order, filter and
// merge rules (:366-425, including its transitionRoot(transition, k) filter
// with the tip index k used as a category index) with those counts.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "runtime.h"

namespace casphy {
namespace tipmerge {

// shared[q] = |N(pj[q]) n N(pk[q])| for ascending lists
__global__ void k_shared(const u32* __restrict__ idx, const u64* __restrict__ off, const u32* __restrict__ cnt,
                         const u32* __restrict__ pj, const u32* __restrict__ pk, u64 npair, u32* __restrict__ shared) {
    const u64 q = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const u32 lane = threadIdx.x & 31;
    if (q >= npair) return;
    const u32 j = pj[q], k = pk[q];
    const u32 nj = cnt[j], nk = cnt[k];
    const u32* a = idx + off[j];
    const u32* b = idx + off[k];
    u32 na = nj, nb = nk;
    if (na > nb) {
        const u32* t = a; a = b; b = t;
        na = nk;
        nb = nj;
    }
    u32 n = 0;
    for (u32 i = lane; i < na; i += 32) {
        const u32 v = a[i];
        u32 lo = 0, hi = nb;
        while (lo < hi) {
            const u32 mid = (lo + hi) >> 1;
            if (b[mid] < v) lo = mid + 1;
            else hi = mid;
        }
        n += lo < nb && b[lo] == v;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xFFFFFFFFu, n, o);
    if (lane == 0) shared[q] = n;
}

}  // namespace tipmerge

namespace {

int root_of(const std::vector<int>& transition, int idx) {
    if (idx == -1) return -1;
    int r = idx;
    while (transition[(size_t)r] != r && transition[(size_t)r] != -1) r = transition[(size_t)r];
    return r;
}

}  // namespace

}  // namespace casphy

extern "C" int casphy_tip_merge(uint32_t ntip, const uint32_t* counts, const uint32_t* idx, double pShared,
                                int32_t* member) {
    using namespace casphy;
    using namespace casphy::tipmerge;
    int rc = require_device();
    if (rc) return rc;
    if (ntip == 0 || !counts || !member) return CASPHY_EINVAL;
    const u32 kCache = 1024u * 128u, kMaxNeighbor = 1024u * 1024u;
    std::vector<u64> off(ntip + 1, 0);
    for (u32 i = 0; i < ntip; i++) {
        if (counts[i] > kMaxNeighbor) {
            casphy_set_last_error_msg("find too many neighbors, increase radius to reduce No. neighbors.");
            return CASPHY_ERANGE;
        }
        off[i + 1] = off[i] + counts[i];
    }
    const u64 total = off[ntip];
    if (total && !idx) return CASPHY_EINVAL;
    // the lists must be ascending, without repeats, inside [0, ntip)
    std::vector<u32> so(ntip);
    std::vector<u64> pairStart(ntip + 1, 0);
    for (u32 i = 0; i < ntip; i++) {
        const u32* l = idx + off[i];
        for (u32 k = 0; k < counts[i]; k++)
            if (l[k] >= ntip || (k && l[k] <= l[k - 1])) {
                casphy_set_last_error_msg("tipMerge: neighbour lists must be ascending row indices");
                return CASPHY_EINVAL;
            }
        u32 j = 0;
        while (j < counts[i] && l[j] <= i) j++;
        so[i] = j;
        pairStart[i + 1] = pairStart[i] + (counts[i] - j);
    }
    const u64 npair = pairStart[ntip];
    std::vector<u32> shared(npair ? npair : 1);
    if (npair) {
        std::vector<u32> pj(npair), pk(npair);
        for (u32 i = 0; i < ntip; i++)
            for (u32 k = so[i]; k < counts[i]; k++) {
                const u64 q = pairStart[i] + (k - so[i]);
                pj[q] = i;
                pk[q] = idx[off[i] + k];
            }
        DeviceScope ds;
        cudaStream_t st = 0;
        auto lay = [&](Carve& c) {
            struct B { u32 *idx, *cnt, *pj, *pk, *sh; u64* off; } b;
            b.idx = c.take<u32>(total);
            b.cnt = c.take<u32>(ntip);
            b.off = c.take<u64>(ntip + 1);
            b.pj = c.take<u32>(npair);
            b.pk = c.take<u32>(npair);
            b.sh = c.take<u32>(npair);
            return b;
        };
        Carve cv;
        lay(cv);
        void* base = nullptr;
        if ((rc = ds.reserve(cv.off + 256, &base))) return rc;
        Carve c2;
        c2.base = static_cast<char*>(base);
        const auto L = lay(c2);
        CASPHY_CUDA_TRY(cudaMemcpyAsync(L.idx, idx, 4ull * total, cudaMemcpyHostToDevice, st));
        CASPHY_CUDA_TRY(cudaMemcpyAsync(L.cnt, counts, 4ull * ntip, cudaMemcpyHostToDevice, st));
        CASPHY_CUDA_TRY(cudaMemcpyAsync(L.off, off.data(), 8ull * (ntip + 1), cudaMemcpyHostToDevice, st));
        CASPHY_CUDA_TRY(cudaMemcpyAsync(L.pj, pj.data(), 4ull * npair, cudaMemcpyHostToDevice, st));
        CASPHY_CUDA_TRY(cudaMemcpyAsync(L.pk, pk.data(), 4ull * npair, cudaMemcpyHostToDevice, st));
        const u64 threads = npair * 32;
        k_shared<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(L.idx, L.off, L.cnt, L.pj, L.pk, npair, L.sh);
        CASPHY_CUDA_TRY(cudaGetLastError());
        CASPHY_CUDA_TRY(cudaMemcpyAsync(shared.data(), L.sh, 4ull * npair, cudaMemcpyDeviceToHost, st));
        CASPHY_CUDA_TRY(cudaStreamSynchronize(st));
    }
    // the reference's visiting order, filter and merge rules
    std::vector<int> transition(ntip, -1);
    std::vector<u32> runPos;
    for (u32 i = 0; i < ntip; i++) member[i] = -1;
    std::vector<u32> search(so);
    int ncat = 0;
    for (u32 c0 = 0; c0 < ntip; c0 += kCache) {
        const u32 c1 = std::min(c0 + kCache, ntip);
        for (u32 j = 0; j < c1; j++) {
            int root1 = member[j];
            if (root1 != -1) root1 = root_of(transition, root1);
            runPos.clear();
            const u32* l = idx + off[j];
            for (u32 k = search[j]; k < counts[j]; k++) {
                const u32 t = l[k];
                if (t >= c1) {
                    search[j] = k;
                    break;
                }
                if (t >= c0 && (root1 == -1 || root1 != root_of(transition, (int)t))) runPos.push_back(k);
            }
            for (u32 k : runPos) {
                const u32 t = l[k];
                const u32 sh = shared[pairStart[j] + (k - so[j])];
                if ((double)sh > counts[j] * pShared || (double)sh > counts[t] * pShared) {
                    const int root2 = root_of(transition, member[t]);
                    if (root1 == -1) {
                        if (root2 == -1) {
                            root1 = ncat;
                            transition[(size_t)ncat] = ncat;
                            member[j] = ncat;
                            member[t] = ncat;
                            ncat++;
                        } else {
                            root1 = root2;
                            member[j] = root2;
                        }
                    } else if (root2 == -1) {
                        member[t] = root1;
                    } else {
                        transition[(size_t)root1] = root2;
                        member[j] = root2;
                        root1 = root2;
                    }
                }
            }
        }
    }
    for (u32 i = 0; i < ntip; i++) member[i] = member[i] == -1 ? ncat++ : root_of(transition, member[i]);
    return CASPHY_OK;
}
