// Batched bootstrap of the bit join with transfer support on B200.
//
// The reference bootstraps by re-running the whole pipeline once per
// replicate from R (vignettes/CasPhy.Rmd:255-291): columns are resampled with
// replacement and, for binary data, handed to joinEdgeBitReverse as integer
// site weights (idx2weight, src/functions.cpp:4485-4492); every replicate tree
// is cut into clades (nodeDesBig, src/functions.cpp:1277-1366) and compared
// with the full-data tree by the transfer distance of TransferDisStream
// (cu/TransferDisStream.cu:22-128); the support of a full-tree clade is the
// fraction of replicates whose normalised distance is <= threshold
// (cal.abs, R/bootstrap_functions.R:190-219).
//
// Here all replicates run in one pass:
//  1. k_bs_prep: one warp per (replicate, tip) gathers the tip's row of the
//     full matrix and builds the replicate's slot matrix and query entries.
//     When every replicate's weights sum to at most the site count (a
//     column resample does), each resampled column is repeated as often as
//     it was drawn (k_bs_gather) and scored with unit weights: the same
//     integer scores and per-column merges as weight w on one column, with
//     one entry per word instead of one per (word, weight bit plane).
//     Otherwise the weights are integer bit planes (the single join's
//     PLANES path).
//  2. k_bs_init: the initial all-pairs scan of every replicate, tiles of all
//     replicates drawn from one queue.
//  3. k_bs_join: persistent and cooperative; each replicate is joined by a
//     group of G co-resident CTAs running the same join engine as the single
//     join (G = 1 needs no barrier beyond the block's own).  G comes from a
//     cost model of the replicate sizes whose constants are fitted to the
//     per-replicate times of the previous call on the device (the
//     autotuner): the largest replicates are split until the longest one no
//     longer outlasts the even share of the work.  Groups run largest first,
//     so every multi-CTA group forms in the first wave.  Member 0 then lays
//     out the replicate tree's post-order (heavier child first, so a walk
//     needs a stack of at most log2(n)+1).
//  4. k_bs_transfer: one thread per (full-tree clade X, replicate).  X is the
//     pre-order tip interval [lo, hi] of the full tree; walking the replicate
//     tree's post-order with a stack of |X n Y| counts gives, for every
//     replicate clade Y, d = |X| + |Y| - 2|X n Y| and the transfer distance
//     min(d, n - d) over the replicate's n tips.  This is the quantity
//     TransferDisStream computes for clade bitsets restricted to the
//     replicate's tips (its pad and group-of-8 arithmetic cancel when no row
//     has bits past the tips), in O(clades x nodes) instead of
//     O(clades x clades x words).
#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "join_bit_model.cuh"
#include "runtime.h"

namespace casphy {
namespace boot {

using namespace bitjoin;
using joinx::kDead;

constexpr u32 kOpInternal = 0x80000000u, kOpRoot = 0x40000000u;
constexpr u32 kXThreads = 128;  // clades per transfer block
constexpr u32 kStack = 32;      // post-order stack (heavier child first: <= log2(n)+1)
constexpr u32 kOpChunk = 2048;  // ops staged in shared memory per step

struct Rep {
    joinx::Common c;
    BitModel<PATH_PLANES>::Args m;
    InitArgs init;
    u32 off;        // first tip in the concatenated cell list
    u32 opsOff;     // first op of this replicate
    u32* ops;       // 2n-1 post-order ops
    u32* eW;
    u32* eQ;
    u32* eLen;
    u32 eStride;
};

// Resampled rows: bit b of word j of (replicate r, tip) is the full row's
// bit colIdx[r][32j+b] (kNone pads).  One warp per (replicate, tip).
__global__ void k_bs_gather(const u32* __restrict__ repOfWarp, const u32* __restrict__ cells,
                            const u32* __restrict__ words, const u32* __restrict__ colIdx, u32 nbin, u32 totalTips,
                            u32* __restrict__ rows) {
    const u32 warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= totalTips) return;
    const u32* src = words + (size_t)cells[warp] * nbin;
    const u32* ci = colIdx + (size_t)repOfWarp[warp] * nbin * 32;
    for (u32 j = lane; j < nbin; j += 32) {
        u32 v = 0;
#pragma unroll 8
        for (u32 b = 0; b < 32; b++) {
            const u32 c = ci[32 * j + b];
            if (c != kNone) v |= ((__ldg(src + (c >> 5)) >> (c & 31)) & 1u) << b;
        }
        rows[(size_t)warp * nbin + j] = v;
    }
}

// One warp per (replicate, tip); rows: the resampled rows by warp, or null
// to read the full rows.
__global__ void k_bs_prep(const Rep* __restrict__ reps, const u32* __restrict__ repOfWarp,
                          const u32* __restrict__ cells, const u32* __restrict__ words, const u32* __restrict__ rows,
                          u32 nbin, u32 totalTips) {
    const u32 warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (warp >= totalTips) return;
    const u32 r = repOfWarp[warp];
    const Rep& R = reps[r];
    const u32 tip = warp - R.off;
    const u32 cell = cells[warp];
    prep_tip(rows ? rows + (size_t)warp * nbin : words + (size_t)cell * nbin, tip, nbin, R.m.nbinP,
             (R.c.ntip + 7u) & ~7u, R.m.nplanes,
             R.m.planeMask, R.m.nodeSeq, R.m.nodeBis, R.m.colT[0], R.eW, R.eQ, R.eLen, R.eStride);
    // initial local maximum: value -1, node ~0 (replaced by the initial scan)
    if ((threadIdx.x & 31) == 0) R.init.initKey[tip] = ((u64)ORD_F32_NEG1 << 32) | 0xFFFFFFFFull;
}

// initial scan: tiles of all replicates from one queue
__global__ void __launch_bounds__(kThreads) k_bs_init(const Rep* __restrict__ reps, const u64* __restrict__ tileStart,
                                                      u32 nrep, unsigned long long* counter) {
    __shared__ unsigned long long s_tile[2];
    __shared__ u64 red[32];
    const u64 total = tileStart[nrep];
    if (threadIdx.x == 0) s_tile[0] = atomicAdd(counter, 1ull);
    __syncthreads();
    int cur = 0;
    for (;;) {
        const u64 t = s_tile[cur];
        if (t >= total) break;
        if (threadIdx.x == 0) s_tile[cur ^ 1] = atomicAdd(counter, 1ull);
        u32 lo = 0, hi = nrep;  // replicate r with tileStart[r] <= t < tileStart[r+1]
        while (hi - lo > 1) {
            const u32 mid = (lo + hi) / 2;
            if (tileStart[mid] <= t) lo = mid;
            else hi = mid;
        }
        init_tile<PATH_PLANES>(reps[lo].init, t - tileStart[lo], red);
        cur ^= 1;
        __syncthreads();
    }
}

// engine slot/node arrays of every replicate: grid (blocks, nrep)
__global__ void k_bs_slot_init(const Rep* __restrict__ reps) {
    const Rep& R = reps[blockIdx.y];
    const joinx::Common& c = R.c;
    const u32 ntip = c.ntip, Sp = (ntip + 7u) & ~7u, nnode = c.nnode;
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < max(Sp, nnode); i += gridDim.x * blockDim.x) {
        if (i < Sp) {
            if (i < ntip) {
                const u64 k = R.init.initKey[i];
                c.lmOrd[0][i] = key_ord(k);
                c.lmIdx[0][i] = key_node(k);
                c.slotNode[0][i] = i;
            } else {
                c.lmOrd[0][i] = c.ordNeg1;
                c.lmIdx[0][i] = 0;
                c.slotNode[0][i] = kDead;
            }
        }
        if (i < 16u * c.nCTA) c.flags[i] = 0u;  // barrier epochs of the replicate's group
        if (i < nnode) {
            c.node2slot[i] = i < ntip ? i : joinx::kNone;
            c.nodeDeath[i] = joinx::kNone;
            c.nodeSize[i] = i < ntip ? 1u : 0u;
        }
    }
}

// Post-order of the replicate tree (raw join edges: node ntip+k has children
// rawEdge[4k+1], rawEdge[4k+3]; the root is 2ntip-2), heavier child first.
// Tip ops carry the tip's full-tree pre-order rank; internal ops carry their
// tip count, the root is flagged.  One thread; offsets in shared memory.
__device__ void build_ops(const joinx::Common& c, const u32* __restrict__ rankOf, u32* ops, u32* s) {
    if (threadIdx.x != 0) return;
    const u32 n = c.ntip;
    if (n == 1) {
        ops[0] = rankOf[0];
        return;
    }
    const u32 root = 2 * n - 2;
    s[root - n] = 0;
    for (u32 v = root + 1; v-- > n;) {
        const u32 k = v - n;
        const u32 base = s[k];
        const u32 tv = c.nodeSize[v];
        ops[base + 2 * tv - 2] = kOpInternal | (v == root ? kOpRoot : 0u) | tv;
        u32 a = c.rawEdge[4 * k + 1], b = c.rawEdge[4 * k + 3];
        u32 ta = c.nodeSize[a], tb = c.nodeSize[b];
        if (tb > ta) {
            const u32 x = a; a = b; b = x;
            const u32 y = ta; ta = tb; tb = y;
        }
        const u32 sb = base + 2 * ta - 1;
        if (a < n) ops[base] = rankOf[a];
        else s[a - n] = base;
        if (b < n) ops[sb] = rankOf[b];
        else s[b - n] = sb;
    }
}

// Work items (replicate, member) in queue order; the members of one
// replicate are consecutive and multi-CTA replicates come first.
template <int PATH>
__global__ void __launch_bounds__(kThreads, 1) k_bs_join(const Rep* __restrict__ reps,
                                                         const u32* __restrict__ itemRep,
                                                         const u32* __restrict__ itemMember, u32 nItem,
                                                         unsigned int* counter, const u32* __restrict__ rankOf) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ u32 s_idx;
    for (;;) {
        if (threadIdx.x == 0) s_idx = atomicAdd(counter, 1u);
        __syncthreads();
        const u32 idx = s_idx;
        __syncthreads();
        if (idx >= nItem) break;
        const u32 r = itemRep[idx], b = itemMember[idx];
        const joinx::Common c = reps[r].c;
        const typename BitModel<PATH>::Args m = reps[r].m;
        const u64 t0 = globaltimer_ns();
        if (c.ntip >= 2) joinx::join_run<BitModel<PATH>>(c, m, b, smem);
        __syncthreads();
        if (b != 0) continue;
        int err = 0;
        if (threadIdx.x == 0) err = *(volatile int*)c.err;
        if (__syncthreads_or(err)) continue;
        build_ops(c, rankOf + reps[r].off, reps[r].ops, reinterpret_cast<u32*>(smem));
        __syncthreads();
        if (threadIdx.x == 0) {
            c.statsOut[6] = t0;
            c.statsOut[7] = globaltimer_ns();
        }
    }
}

// Transfer distances: grid (clade blocks, replicates).
struct XferArgs {
    u32 nX, nrep, fill;
    const u32* Xlo;
    const u32* Xhi;
    const u32* repN;       // tips per replicate
    const u32* repOff;     // first tip (sorted ranks) per replicate
    const u32* repOpsOff;  // first op per replicate
    const u32* sortedRank;
    const u32* ops;
    double threshold;
    u32* ymin;   // nrep x nX
    u32* ysize;  // nrep x nX
    u32* support;
    int* err;
};

__device__ __forceinline__ u32 lower_bound_u32(const u32* a, u32 n, u32 v) {
    u32 lo = 0, hi = n;
    while (lo < hi) {
        const u32 mid = (lo + hi) >> 1;
        if (a[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(kXThreads) k_bs_transfer(XferArgs a) {
    __shared__ u32 stack[kStack * kXThreads];
    __shared__ u32 sops[kOpChunk];
    const u32 r = blockIdx.y;
    const u32 x = blockIdx.x * kXThreads + threadIdx.x;
    const bool ok = x < a.nX;
    const u32 n = a.repN[r];
    const u32* srt = a.sortedRank + a.repOff[r];
    const u32* ops = a.ops + a.repOpsOff[r];
    const u32 lo = ok ? a.Xlo[x] : 1u, hi = ok ? a.Xhi[x] : 0u;
    const u32 nX = ok ? lower_bound_u32(srt, n, hi + 1) - lower_bound_u32(srt, n, lo) : 0u;
    u32 best = a.fill;
    u32 sp = 0;
    bool over = false;
    const u32 nops = 2 * n - 1;
    for (u32 o0 = 0; o0 < nops; o0 += kOpChunk) {
        const u32 m = min(kOpChunk, nops - o0);
        __syncthreads();
        for (u32 i = threadIdx.x; i < m; i += kXThreads) sops[i] = ops[o0 + i];
        __syncthreads();
        for (u32 i = 0; i < m; i++) {
            const u32 op = sops[i];
            if (!(op & kOpInternal)) {
                if (sp < kStack) stack[sp * kXThreads + threadIdx.x] = (op >= lo && op <= hi) ? 1u : 0u;
                else over = true;
                sp++;
            } else {
                if (sp < 2 || sp > kStack) {
                    over = true;
                    continue;
                }
                const u32 cnt = stack[(sp - 1) * kXThreads + threadIdx.x] + stack[(sp - 2) * kXThreads + threadIdx.x];
                sp--;
                stack[(sp - 1) * kXThreads + threadIdx.x] = cnt;
                if (!(op & kOpRoot)) {
                    const u32 sY = op & 0x3FFFFFFFu;
                    const u32 d = nX + sY - 2 * cnt;
                    const u32 t = min(d, n - d);
                    best = min(best, t);
                }
            }
        }
    }
    if (over && threadIdx.x == 0) atomicCAS(a.err, 0, CASPHY_EINTERNAL);
    if (!ok) return;
    const u32 ys = min(nX, n - nX);
    a.ymin[(size_t)r * a.nX + x] = best;
    a.ysize[(size_t)r * a.nX + x] = ys;
    if (ys > 0 && (double)best <= a.threshold * (double)ys) atomicAdd(a.support + x, 1u);
}

}  // namespace boot

using namespace boot;

static int full_tree_intervals(u32 ntip, const u32* edge, std::vector<u32>& Xlo, std::vector<u32>& Xhi,
                               std::vector<u32>& rank) {
    const u32 nn = 2 * ntip - 1, nedge = 2 * ntip - 2, none = 0xFFFFFFFFu;
    std::vector<u32> kidA(nn, none), kidB(nn, none);
    std::vector<unsigned char> isChild(nn, 0);
    for (u32 e = 0; e < nedge; e++) {
        const u32 p = edge[2 * e], c = edge[2 * e + 1];
        if (p >= nn || c >= nn || p < ntip || isChild[c]) return CASPHY_EINVAL;
        isChild[c] = 1;
        if (kidA[p] == none) kidA[p] = c;
        else if (kidB[p] == none) kidB[p] = c;
        else return CASPHY_EINVAL;
    }
    u32 root = none, nroot = 0;
    for (u32 v = 0; v < nn; v++)
        if (!isChild[v]) {
            root = v;
            nroot++;
        }
    if (nroot != 1 || root < ntip) return CASPHY_EINVAL;
    rank.assign(ntip, none);
    std::vector<u32> lo(nn, none), hi(nn, 0), stack{root}, post;
    post.reserve(nn);
    u32 next = 0;
    while (!stack.empty()) {
        const u32 v = stack.back();
        stack.pop_back();
        post.push_back(v);
        if (v < ntip) {
            rank[v] = next++;
        } else {
            if (kidB[v] == none) return CASPHY_EINVAL;
            stack.push_back(kidB[v]);
            stack.push_back(kidA[v]);
        }
        if (post.size() > nn) return CASPHY_EINVAL;
    }
    if (post.size() != nn || next != ntip) return CASPHY_EINVAL;
    for (auto it = post.rbegin(); it != post.rend(); ++it) {
        const u32 v = *it;
        if (v < ntip) {
            lo[v] = hi[v] = rank[v];
        } else {
            lo[v] = std::min(lo[kidA[v]], lo[kidB[v]]);
            hi[v] = std::max(hi[kidA[v]], hi[kidB[v]]);
        }
    }
    Xlo.clear();
    Xhi.clear();
    for (u32 v = ntip; v < nn; v++) {
        if (v == root) continue;
        Xlo.push_back(lo[v]);
        Xhi.push_back(hi[v]);
    }
    return CASPHY_OK;
}

}  // namespace casphy

namespace casphy {
namespace boot {

// Cost of joining one replicate of n cells with G CTAs: its phases times
// (alpha + beta * n / G + gamma when G > 1) -- a fixed per-phase part, the
// scan of the slots each CTA owns, and the cross-CTA barrier.  The constants
// start from a B200 estimate and are refitted on every call from the
// measured replicate times, per device.
struct Tune {
    int measured = 0;
    double alpha = 6.0;        // us per phase
    double beta = 1.8e-3;      // us per phase per slot of a CTA
    double gamma = 2.0;        // us per phase for the barrier of a group
    double phasesPerTip = 1.7;
};
constexpr int kMaxDev = 64;
constexpr u32 kMaxGroup = 8;
Tune g_tune[kMaxDev];  // read and written under the device's workspace lock

inline double cost_us(const Tune& T, u32 n, u32 G) {
    return T.phasesPerTip * n * (T.alpha + T.beta * (double)n / G + (G > 1 ? T.gamma : 0.0));
}

// CTAs per replicate: split the replicate with the longest predicted join
// while it outlasts the even share of all work over `slots` CTAs and a split
// still shortens it.
std::vector<u32> split_groups(const Tune& T, const std::vector<u32>& repN, u32 slots) {
    const u32 nrep = (u32)repN.size();
    std::vector<u32> G(nrep, 1);
    // CASPHY_BS_GROUP=g fixes g CTAs for every replicate of 512 cells or
    // more while they fit the SMs (the cost model is bypassed)
    if (const char* env = std::getenv("CASPHY_BS_GROUP")) {
        const u32 g = std::min<u32>((u32)std::max(1, std::atoi(env)), kMaxGroup);
        u32 used = 0;
        for (u32 r = 0; r < nrep; r++)
            if (g > 1 && repN[r] >= 512 && used + g <= slots) {
                G[r] = g;
                used += g;
            }
        return G;
    }
    std::vector<double> t(nrep);
    double W = 0;
    for (u32 r = 0; r < nrep; r++) {
        t[r] = cost_us(T, repN[r], 1);
        W += t[r];
    }
    u32 inGroups = 0;
    for (;;) {
        u32 rm = 0;
        for (u32 r = 1; r < nrep; r++)
            if (t[r] > t[rm]) rm = r;
        if (t[rm] <= W / slots || G[rm] >= kMaxGroup || repN[rm] < 512) break;
        const u32 g = G[rm] + 1, extra = G[rm] == 1 ? 2 : 1;
        const double tn = cost_us(T, repN[rm], g);
        if (tn >= t[rm] || inGroups + extra > slots) break;
        W += tn * g - t[rm] * G[rm];
        inGroups += extra;
        G[rm] = g;
        t[rm] = tn;
    }
    return G;
}

// Refit alpha and beta on the single-CTA replicates and gamma on the
// groups, by least squares of the per-phase time; keeps the previous value
// of a constant the measurements cannot pin down.
void refit(Tune& T, const std::vector<u32>& repN, const std::vector<u32>& G, const std::vector<double>& us,
           const std::vector<unsigned long long>& phases) {
    double s1 = 0, sx = 0, sxx = 0, sy = 0, sxy = 0, ptot = 0, ntot = 0;
    for (size_t r = 0; r < repN.size(); r++) {
        if (phases[r] == 0 || us[r] <= 0) continue;
        ptot += (double)phases[r];
        ntot += repN[r];
        if (G[r] != 1) continue;
        const double x = repN[r], y = us[r] / (double)phases[r];
        s1 += 1;
        sx += x;
        sxx += x * x;
        sy += y;
        sxy += x * y;
    }
    if (ntot > 0) T.phasesPerTip = ptot / ntot;
    const double det = s1 * sxx - sx * sx;
    if (s1 >= 8 && det > 0) {
        const double b = (s1 * sxy - sx * sy) / det, a = (sy - b * sx) / s1;
        if (a > 0 && b > 0) {
            T.alpha = a;
            T.beta = b;
            T.measured = 1;
        }
    }
    double gs = 0, gn = 0;
    for (size_t r = 0; r < repN.size(); r++) {
        if (G[r] == 1 || phases[r] == 0 || us[r] <= 0) continue;
        gs += us[r] / (double)phases[r] - T.alpha - T.beta * repN[r] / G[r];
        gn += 1;
    }
    if (gn > 0) T.gamma = std::max(0.1, gs / gn);
}

}  // namespace boot
}  // namespace casphy

extern "C" int casphy_bootstrap_bit(uint32_t ntip, uint32_t nbin, const uint32_t* words, const uint32_t* full_edge,
                                    uint32_t nrep, const uint32_t* rep_offsets, const uint32_t* rep_cells,
                                    const double* rep_weights, int ancestralType, double threshold,
                                    uint32_t* support, uint32_t* ymin_out, uint32_t* ysize_out,
                                    uint32_t* rep_raw_edges, casphy_bootstrap_stats* stats) {
    using namespace casphy;
    int rc = require_device();
    if (rc) return rc;
    if (ntip < 3 || nbin == 0 || nbin > kMaxBin || !words || !full_edge || nrep == 0 || !rep_offsets || !rep_cells ||
        !rep_weights || !support || !(threshold >= 0)) {
        casphy_set_last_error_msg("bootstrap: bad arguments");
        return CASPHY_EINVAL;
    }
    std::vector<u32> Xlo, Xhi, rank;
    if ((rc = full_tree_intervals(ntip, full_edge, Xlo, Xhi, rank))) {
        casphy_set_last_error_msg("bootstrap: full_edge is not a binary tree over ntip tips");
        return rc;
    }
    const u32 nX = (u32)Xlo.size(), nsite = nbin * 32, nbinP = (nbin + 3u) & ~3u;
    // replicate sizes, weights -> bit planes
    std::vector<u32> repN(nrep), repOpsOff(nrep + 1, 0), nplanesOf(nrep);
    u32 nmax = 0, totalTips = rep_offsets[nrep] - rep_offsets[0];
    if (rep_offsets[0] != 0) return CASPHY_EINVAL;
    u32 P = 1;
    for (u32 r = 0; r < nrep; r++) {
        if (rep_offsets[r + 1] < rep_offsets[r]) return CASPHY_EINVAL;
        repN[r] = rep_offsets[r + 1] - rep_offsets[r];
        if (repN[r] < 2) {
            casphy_set_last_error_msg("bootstrap: every replicate needs at least 2 cells");
            return CASPHY_EINVAL;
        }
        nmax = std::max(nmax, repN[r]);
        repOpsOff[r + 1] = repOpsOff[r] + 2 * repN[r] - 1;
        double tot = 0;
        u32 maxw = 0;
        for (u32 i = 0; i < nsite; i++) {
            const double w = rep_weights[(size_t)r * nsite + i];
            if (!(w >= 0) || w != std::floor(w) || w >= 16777216.0) {
                casphy_set_last_error_msg("bootstrap: replicate weights must be non-negative integers");
                return CASPHY_EINVAL;
            }
            tot += w;
            maxw = std::max(maxw, (u32)w);
        }
        if (tot > 16777216.0) return CASPHY_ERANGE;
        u32 np = 0;
        while ((1u << np) <= maxw && np < 24) np++;
        P = std::max(P, std::max(np, 1u));
    }
    for (u32 i = 0; i < totalTips; i++)
        if (rep_cells[i] >= ntip) return CASPHY_EINVAL;
    // repeated columns when every replicate's draws fit the row, else planes
    bool repeat = true;
    for (u32 r = 0; r < nrep && repeat; r++) {
        double tot = 0;
        for (u32 i = 0; i < nsite; i++) tot += rep_weights[(size_t)r * nsite + i];
        repeat = tot <= (double)nsite;
    }
    std::vector<u32> colIdx;
    if (repeat) {
        P = 1;
        colIdx.assign((size_t)nrep * nsite, joinx::kNone);
        for (u32 r = 0; r < nrep; r++) {
            size_t pos = (size_t)r * nsite;
            for (u32 i = 0; i < nsite; i++)
                for (u32 c = (u32)rep_weights[(size_t)r * nsite + i]; c > 0; c--) colIdx[pos++] = i;
        }
    }
    const u32 nplanes = repeat ? 0u : P;
    std::vector<u32> planes((size_t)nrep * P * nbin, 0u);
    if (!repeat)
        for (u32 r = 0; r < nrep; r++)
            for (u32 i = 0; i < nsite; i++) {
                const u32 v = (u32)rep_weights[(size_t)r * nsite + i];
                for (u32 k = 0; k < P; k++)
                    if ((v >> k) & 1u) planes[((size_t)r * P + k) * nbin + i / 32] |= 1u << (i % 32);
            }
    const u32 eStride = nbin * P;
    // per-replicate layout in one arena
    DeviceScope ds;
    int nSM = 0;
    CASPHY_CUDA_TRY(cudaDeviceGetAttribute(&nSM, cudaDevAttrMultiProcessorCount, ds.dev));
    // CTAs per replicate from the device's cost model (one join CTA per SM)
    boot::Tune& tune = boot::g_tune[(ds.dev >= 0 && ds.dev < boot::kMaxDev) ? ds.dev : 0];
    const int tunedBefore = tune.measured;
    std::vector<u32> Gs = boot::split_groups(tune, repN, (u32)nSM);
    u32 nItemAll = 0;
    for (u32 g : Gs) nItemAll += g;
    struct RepBufs {
        u32 *planeMask, *nodeSeq, *nodeBis, *colT0, *colT1, *lm[6], *node2slot, *nodeDeath, *nodeSize, *rawEdge;
        u32 *eW, *eQ, *eLen, *pubCnt, *counts, *flags;
        unsigned long long* initKey;
        joinx::BlockRec* pub;
        u64* partial;
        u64* chunkStart;
        unsigned long long* stats;
    };
    auto rep_layout = [&](Carve& c, u32 n, u32 G) {
        RepBufs b;
        const u32 Sp = (n + 7u) & ~7u, nnode = 2 * n - 1, nChunks = (n + kCap - 1) / kCap;
        b.planeMask = c.take<u32>((size_t)P * nbin);
        b.nodeSeq = c.take<u32>((size_t)nnode * nbinP);
        b.nodeBis = c.take<u32>((size_t)nnode * nbinP);
        b.colT0 = c.take<u32>((size_t)nbin * Sp);
        b.colT1 = c.take<u32>((size_t)nbin * Sp);
        for (int i = 0; i < 6; i++) b.lm[i] = c.take<u32>(Sp);
        b.node2slot = c.take<u32>(nnode);
        b.nodeDeath = c.take<u32>(nnode);
        b.nodeSize = c.take<u32>(nnode);
        b.rawEdge = c.take<u32>((size_t)4 * n);
        b.eW = c.take<u32>((size_t)n * eStride);
        b.eQ = c.take<u32>((size_t)n * eStride);
        b.eLen = c.take<u32>(n);
        b.initKey = c.take<unsigned long long>(n);
        b.pub = c.take<joinx::BlockRec>(4 * G);
        b.pubCnt = c.take<u32>(2 * G);
        b.partial = c.take<u64>((size_t)2 * G * joinx::kMaxBatch);
        b.counts = c.take<u32>(G);
        b.flags = c.take<u32>(16 * G);
        b.chunkStart = c.take<u64>(nChunks + 1);
        b.stats = c.take<unsigned long long>(8);
        return b;
    };
    struct Glob {
        Rep* reps;
        u32 *repOfWarp, *cells, *words, *itemRep, *itemMember, *rankOf, *sortedRank, *ops, *Xlo, *Xhi, *repN, *repOff, *repOpsOff;
        u32 *ymin, *ysize, *support;
        u64* tileStart;
        unsigned long long* counter;
        unsigned int* jcounter;
        int* errs;
        int* xerr;
        u32* colIdx;
        u32* rrows;
    };
    auto glob_layout = [&](Carve& c) {
        Glob g;
        g.reps = c.take<Rep>(nrep);
        g.repOfWarp = c.take<u32>(totalTips);
        g.cells = c.take<u32>(totalTips);
        g.words = c.take<u32>((size_t)ntip * nbin);
        g.itemRep = c.take<u32>(nItemAll);
        g.itemMember = c.take<u32>(nItemAll);
        g.rankOf = c.take<u32>(totalTips);
        g.sortedRank = c.take<u32>(totalTips);
        g.ops = c.take<u32>(repOpsOff[nrep]);
        g.Xlo = c.take<u32>(nX);
        g.Xhi = c.take<u32>(nX);
        g.repN = c.take<u32>(nrep);
        g.repOff = c.take<u32>(nrep);
        g.repOpsOff = c.take<u32>(nrep);
        g.ymin = c.take<u32>((size_t)nrep * nX);
        g.ysize = c.take<u32>((size_t)nrep * nX);
        g.support = c.take<u32>(nX);
        g.tileStart = c.take<u64>(nrep + 1);
        g.counter = c.take<unsigned long long>(1);
        g.jcounter = c.take<unsigned int>(1);
        g.errs = c.take<int>(nrep);
        g.xerr = c.take<int>(1);
        g.colIdx = c.take<u32>(repeat ? (size_t)nrep * nsite : 1);
        g.rrows = c.take<u32>(repeat ? (size_t)totalTips * nbin : 1);
        return g;
    };
    Carve cv;
    glob_layout(cv);
    for (u32 r = 0; r < nrep; r++) rep_layout(cv, repN[r], Gs[r]);
    void* base = nullptr;
    if ((rc = ds.reserve(cv.off + 256, &base))) return rc;
    Carve c2;
    c2.base = static_cast<char*>(base);
    const Glob G = glob_layout(c2);
    std::vector<Rep> reps(nrep);
    std::vector<RepBufs> rb(nrep);
    std::vector<u64> tileStart(nrep + 1, 0), chunkAll;
    std::vector<std::vector<u64>> chunkStarts(nrep);
    for (u32 r = 0; r < nrep; r++) {
        rb[r] = rep_layout(c2, repN[r], Gs[r]);
        const u32 n = repN[r], Sp = (n + 7u) & ~7u, nChunks = (n + kCap - 1) / kCap;
        auto& cs = chunkStarts[r];
        cs.assign(nChunks + 1, 0);
        for (u32 k = 0; k < nChunks; k++) {
            const u64 end = std::min<u64>((u64)(k + 1) * kCap, n);
            cs[k + 1] = cs[k] + (end >= 1 ? end - 1 : 0);
        }
        tileStart[r + 1] = tileStart[r] + cs[nChunks];
        Rep& R = reps[r];
        std::memset(&R, 0, sizeof(Rep));
        joinx::Common& c = R.c;
        const RepBufs& b = rb[r];
        c.ntip = n; c.nnode = 2 * n - 1; c.nCTA = Gs[r]; c.align = 8;
        c.lmOrd[0] = b.lm[0]; c.lmIdx[0] = b.lm[1]; c.slotNode[0] = b.lm[2];
        c.lmOrd[1] = b.lm[3]; c.lmIdx[1] = b.lm[4]; c.slotNode[1] = b.lm[5];
        c.node2slot = b.node2slot; c.nodeDeath = b.nodeDeath; c.nodeSize = b.nodeSize; c.rawEdge = b.rawEdge;
        c.pub = b.pub; c.pubCnt = b.pubCnt; c.partial = b.partial; c.counts = b.counts; c.flags = b.flags;
        c.err = G.errs + r; c.limitNs = 20ull * 1000 * 1000 * 1000; c.statsOut = b.stats;
        c.Rmax = ((n + Gs[r] - 1) / Gs[r] + 7u) & ~7u; c.ordNeg1 = ORD_F32_NEG1; c.compactMin = 4096; c.compactQ8 = 192; c.bytesPerPairSite = 4000;
        c.prof = nullptr;
        c.maxBatch = joinx::stale_batch_setting();
        c.deathWords = (2 * n - 1 + 31) / 32;  // joined-node bitmap: 2.5 KB at 10,000 cells
        c.keepSizes = 1;                         // build_ops lays out clades by node size
        R.m = BitModel<PATH_PLANES>::Args{nbin, nbinP, nplanes, ancestralType ? 1 : 0, b.planeMask, nullptr,
                                          b.nodeSeq, b.nodeBis, {b.colT0, b.colT1}};
        R.init = InitArgs{n, nbin, Sp, eStride, b.colT0, b.eW, b.eQ, b.eLen, nullptr, b.chunkStart, nChunks,
                          cs[nChunks], nullptr, b.initKey};
        R.off = rep_offsets[r];
        R.opsOff = repOpsOff[r];
        R.ops = G.ops + repOpsOff[r];
        R.eW = b.eW; R.eQ = b.eQ; R.eLen = b.eLen; R.eStride = eStride;
    }
    // host tables: replicate of each tip, ranks, sorted ranks, largest-first order
    std::vector<u32> repOfWarp(totalTips), rankOf(totalTips), sortedRank(totalTips), order(nrep), repOff(nrep);
    for (u32 r = 0; r < nrep; r++) {
        repOff[r] = rep_offsets[r];
        for (u32 i = rep_offsets[r]; i < rep_offsets[r + 1]; i++) {
            repOfWarp[i] = r;
            rankOf[i] = rank[rep_cells[i]];
        }
        std::copy(rankOf.begin() + rep_offsets[r], rankOf.begin() + rep_offsets[r + 1], sortedRank.begin() + rep_offsets[r]);
        std::sort(sortedRank.begin() + rep_offsets[r], sortedRank.begin() + rep_offsets[r + 1]);
        for (u32 i = rep_offsets[r] + 1; i < rep_offsets[r + 1]; i++)
            if (sortedRank[i] == sortedRank[i - 1]) {
                casphy_set_last_error_msg("bootstrap: a replicate lists a cell twice");
                return CASPHY_EINVAL;
            }
    }
    // join items: groups first, then the largest replicates first
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(),
                     [&](u32 a, u32 b) { return Gs[a] != Gs[b] ? Gs[a] > Gs[b] : repN[a] > repN[b]; });
    std::vector<u32> itemRep, itemMember;
    u32 maxG = 1, inGroups = 0;
    for (u32 r : order) {
        for (u32 b = 0; b < Gs[r]; b++) {
            itemRep.push_back(r);
            itemMember.push_back(b);
        }
        maxG = std::max(maxG, Gs[r]);
        if (Gs[r] > 1) inGroups += Gs[r];
    }
    const u32 nItem = (u32)itemRep.size();
    // shared memory of a join CTA: engine + model, or the post-order offsets
    using M = BitModel<PATH_PLANES>;
    int maxSmem = 0;
    CASPHY_CUDA_TRY(cudaDeviceGetAttribute(&maxSmem, cudaDevAttrMaxSharedMemoryPerBlockOptin, ds.dev));
    auto joinSmem = [&] {
        size_t m = 0;
        for (u32 r = 0; r < nrep; r++)
            m = std::max(m, M::engine_smem_bytes(Gs[r], reps[r].c.Rmax, reps[r].c.deathWords) +
                                M::model_smem_bytes(reps[r].m));
        return m;
    };
    size_t smemJoin = joinSmem();
    if (smemJoin + 1024 > (size_t)maxSmem) {  // without the joined-node bitmaps (node deaths from global memory)
        for (u32 r = 0; r < nrep; r++) reps[r].c.deathWords = 0;
        smemJoin = joinSmem();
    }
    const size_t smem = std::max(smemJoin, (size_t)4 * nmax);
    if (smem + 1024 > (size_t)maxSmem) {
        casphy_set_last_error_msg("bootstrap: replicate too large for one CTA's shared memory");
        return CASPHY_ERANGE;
    }
    cudaStream_t st = 0;
    cudaEvent_t ev[4];
    for (auto& e : ev) CASPHY_CUDA_TRY(cudaEventCreate(&e));
    auto up = [&](void* d, const void* h, size_t n) { return cudaMemcpyAsync(d, h, n, cudaMemcpyHostToDevice, st); };
    // per-replicate plane masks and tile tables
    for (u32 r = 0; r < nrep; r++) {
        const RepBufs& b = rb[r];
        const u32 nChunks = (u32)chunkStarts[r].size() - 1;
        CASPHY_CUDA_TRY(up(b.planeMask, planes.data() + (size_t)r * P * nbin, sizeof(u32) * P * nbin));
        CASPHY_CUDA_TRY(up(b.chunkStart, chunkStarts[r].data(), sizeof(u64) * (nChunks + 1)));
    }
    CASPHY_CUDA_TRY(up(G.reps, reps.data(), sizeof(Rep) * nrep));
    CASPHY_CUDA_TRY(up(G.repOfWarp, repOfWarp.data(), 4ull * totalTips));
    CASPHY_CUDA_TRY(up(G.cells, rep_cells, 4ull * totalTips));
    CASPHY_CUDA_TRY(up(G.words, words, 4ull * ntip * nbin));
    CASPHY_CUDA_TRY(up(G.itemRep, itemRep.data(), 4ull * nItem));
    CASPHY_CUDA_TRY(up(G.itemMember, itemMember.data(), 4ull * nItem));
    CASPHY_CUDA_TRY(up(G.rankOf, rankOf.data(), 4ull * totalTips));
    CASPHY_CUDA_TRY(up(G.sortedRank, sortedRank.data(), 4ull * totalTips));
    CASPHY_CUDA_TRY(up(G.Xlo, Xlo.data(), 4ull * nX));
    CASPHY_CUDA_TRY(up(G.Xhi, Xhi.data(), 4ull * nX));
    CASPHY_CUDA_TRY(up(G.repN, repN.data(), 4ull * nrep));
    CASPHY_CUDA_TRY(up(G.repOff, repOff.data(), 4ull * nrep));
    CASPHY_CUDA_TRY(up(G.repOpsOff, repOpsOff.data(), 4ull * nrep));
    CASPHY_CUDA_TRY(up(G.tileStart, tileStart.data(), 8ull * (nrep + 1)));
    CASPHY_CUDA_TRY(cudaMemsetAsync(G.support, 0, 4ull * nX, st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(G.counter, 0, sizeof(unsigned long long), st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(G.jcounter, 0, sizeof(unsigned int), st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(G.errs, 0, sizeof(int) * nrep, st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(G.xerr, 0, sizeof(int), st));
    if (repeat) CASPHY_CUDA_TRY(up(G.colIdx, colIdx.data(), 4ull * nrep * nsite));
    int perSM = 0;
    CASPHY_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_bs_init, kThreads, 0));
    void* joinFn = (void*)k_bs_join<PATH_PLANES>;
    CASPHY_CUDA_TRY(cudaFuncSetAttribute(joinFn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per = 0;
    CASPHY_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, joinFn, kThreads, smem));
    if (per < 1) return CASPHY_ERANGE;
    const u32 joinGrid = std::min<u32>(nItem, (u32)(nSM * per));
    if (inGroups > joinGrid) return CASPHY_EINTERNAL;  // a group could not form
    const Rep* a0 = G.reps;
    const u32* a1 = G.itemRep;
    const u32* a2 = G.itemMember;
    u32 a3 = nItem;
    unsigned int* a4 = G.jcounter;
    const u32* a5 = G.rankOf;
    void* joinArgs[] = {(void*)&a0, (void*)&a1, (void*)&a2, (void*)&a3, (void*)&a4, (void*)&a5};
    XferArgs xa{nX, nrep, 32u * ((ntip + 31) / 32), G.Xlo, G.Xhi, G.repN, G.repOff, G.repOpsOff, G.sortedRank, G.ops,
                threshold, G.ymin, G.ysize, G.support, G.xerr};
    // the whole pass: prep, initial scans, the persistent cooperative join
    // (every CTA resident, so each group's members run together), transfer
    const u64 launches = (repeat ? 1 : 0) + 5;
    auto enqueue = [&](cudaStream_t s) -> cudaError_t {
        cudaError_t e;
        if ((e = cudaEventRecordWithFlags(ev[0], s, cudaEventRecordExternal)) != cudaSuccess) return e;
        if (repeat)
            k_bs_gather<<<(totalTips + 7) / 8, 256, 0, s>>>(G.repOfWarp, G.cells, G.words, G.colIdx, nbin, totalTips,
                                                          G.rrows);
        k_bs_prep<<<(totalTips + 7) / 8, 256, 0, s>>>(G.reps, G.repOfWarp, G.cells, G.words,
                                                      repeat ? G.rrows : nullptr, nbin, totalTips);
        k_bs_init<<<nSM * std::max(perSM, 1), kThreads, 0, s>>>(G.reps, G.tileStart, nrep, G.counter);
        k_bs_slot_init<<<dim3((2 * nmax + 255) / 256, nrep), 256, 0, s>>>(G.reps);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if ((e = cudaEventRecordWithFlags(ev[1], s, cudaEventRecordExternal)) != cudaSuccess) return e;
        if ((e = cudaLaunchCooperativeKernel(joinFn, dim3(joinGrid), dim3(kThreads), joinArgs, smem, s)) !=
            cudaSuccess)
            return e;
        if ((e = cudaEventRecordWithFlags(ev[2], s, cudaEventRecordExternal)) != cudaSuccess) return e;
        k_bs_transfer<<<dim3((nX + kXThreads - 1) / kXThreads, nrep), kXThreads, 0, s>>>(xa);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        return cudaEventRecordWithFlags(ev[3], s, cudaEventRecordExternal);
    };
    // run it as one captured CUDA graph; launch directly if capture fails
    CASPHY_CUDA_TRY(cudaStreamSynchronize(st));
    bool graphed = false;
    {
        cudaStream_t cs = nullptr;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            const cudaError_t e = enqueue(cs);
            const cudaError_t e2 = cudaStreamEndCapture(cs, &graph);
            if (e == cudaSuccess && e2 == cudaSuccess && graph && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess)
                graphed = cudaGraphLaunch(exec, cs) == cudaSuccess && cudaStreamSynchronize(cs) == cudaSuccess;
        }
        if (!graphed) cudaGetLastError();  // a refused capture is not an error of the call
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (cs) cudaStreamDestroy(cs);
    }
    if (!graphed) CASPHY_CUDA_TRY(enqueue(st));
    std::vector<int> errs(nrep);
    int xerr = 0;
    CASPHY_CUDA_TRY(cudaMemcpyAsync(errs.data(), G.errs, sizeof(int) * nrep, cudaMemcpyDeviceToHost, st));
    CASPHY_CUDA_TRY(cudaMemcpyAsync(&xerr, G.xerr, sizeof(int), cudaMemcpyDeviceToHost, st));
    CASPHY_CUDA_TRY(cudaMemcpyAsync(support, G.support, 4ull * nX, cudaMemcpyDeviceToHost, st));
    if (ymin_out) CASPHY_CUDA_TRY(cudaMemcpyAsync(ymin_out, G.ymin, 4ull * nrep * nX, cudaMemcpyDeviceToHost, st));
    if (ysize_out) CASPHY_CUDA_TRY(cudaMemcpyAsync(ysize_out, G.ysize, 4ull * nrep * nX, cudaMemcpyDeviceToHost, st));
    if (rep_raw_edges) {
        size_t o = 0;
        for (u32 r = 0; r < nrep; r++) {
            const size_t ne = (size_t)4 * (repN[r] - 1);
            CASPHY_CUDA_TRY(cudaMemcpyAsync(rep_raw_edges + o, rb[r].rawEdge, 4 * ne, cudaMemcpyDeviceToHost, st));
            o += ne;
        }
    }
    std::vector<unsigned long long> hst((size_t)8 * nrep);
    for (u32 r = 0; r < nrep; r++)
        CASPHY_CUDA_TRY(cudaMemcpyAsync(hst.data() + 8 * r, rb[r].stats, sizeof(unsigned long long) * 8,
                                        cudaMemcpyDeviceToHost, st));
    CASPHY_CUDA_TRY(cudaStreamSynchronize(st));
    unsigned long long phases = 0;
    std::vector<double> repUs(nrep, 0.0);
    std::vector<unsigned long long> repPhases(nrep, 0);
    double longest = 0, busy = 0;
    for (u32 r = 0; r < nrep; r++) {
        phases += hst[8 * r + 3];
        repPhases[r] = hst[8 * r + 3];
        const unsigned long long t0 = hst[8 * r + 6], t1 = hst[8 * r + 7];
        repUs[r] = t1 > t0 ? (double)(t1 - t0) * 1e-3 : 0.0;
        longest = std::max(longest, repUs[r]);
        busy += repUs[r] * Gs[r];
    }
    for (u32 r = 0; r < nrep; r++)
        if (errs[r]) {
            casphy_set_last_error_msg(errs[r] == CASPHY_ETIMEOUT ? "bootstrap: a replicate join timed out"
                                                                  : "bootstrap: a replicate join failed");
            return errs[r];
        }
    if (xerr) {
        casphy_set_last_error_msg("bootstrap: post-order stack overflow");
        return CASPHY_EINTERNAL;
    }
    boot::refit(tune, repN, Gs, repUs, repPhases);
    float tInit = 0, tJoin = 0, tX = 0, tAll = 0;
    cudaEventElapsedTime(&tInit, ev[0], ev[1]);
    cudaEventElapsedTime(&tJoin, ev[1], ev[2]);
    cudaEventElapsedTime(&tX, ev[2], ev[3]);
    cudaEventElapsedTime(&tAll, ev[0], ev[3]);
    for (auto& e : ev) cudaEventDestroy(e);
    if (stats) {
        casphy_bootstrap_stats s{};
        s.nrep = nrep;
        s.nclade = nX;
        s.prep_ms = tInit;
        s.join_ms = tJoin;
        s.transfer_ms = tX;
        s.total_ms = tAll;
        s.kernel_launches = launches;
        s.join_phases = phases;
        s.max_ctas_per_rep = maxG;
        s.graph = graphed ? 1u : 0u;
        s.tuned = tunedBefore ? 1u : 0u;
        s.join_longest_ms = longest * 1e-3;
        s.join_busy_ms = busy * 1e-3;
        s.cost_alpha_us = tune.alpha;
        s.cost_beta_us = tune.beta;
        s.cost_gamma_us = tune.gamma;
        *stats = s;
    }
    return CASPHY_OK;
}
