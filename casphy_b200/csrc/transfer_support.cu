// Clade matching of query trees against a reference tree on B200: the
// reference's approximateCompare2_AVX2 (src/functions.cpp:5450-5600) batched
// over all query trees, and the transfer support cal.abs builds from it
// (R/bootstrap_functions.R:190-219).
//
// The reference visits one query tree's edges in reverse order.  An internal
// child d ORs its tip set into its parent's and then walks up the reference
// tree from the stop node of each of its children; at each reference node it
// takes the XOR distance to d and the count of tips outside d, lowers that
// node's best distance (ties go to the d visited later) and d's best (ties go
// to the node reached later, which becomes d's stop node).  The only links
// between different d are the children's stop nodes and the reference nodes'
// best distances.  So here all nodes of one height, across all query trees,
// are searched at once (one warp each, heights in increasing order, so a
// node's children are done before it), and a reference node's best is kept
// as one 64-bit key (distance, then the complement of d's visiting rank)
// lowered with atomicMin, which gives the same minimum and the same winner
// of every tie whatever order the warps run in.  The open-row cache of the
// reference (8192 rows) only decides whether the function runs out of cache;
// the host replays it per tree.
#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

#include "common.cuh"
#include "runtime.h"

namespace casphy {
namespace tsup {

constexpr u32 kThreads = 256;

struct Item {
    u32 tree, node;  // node = internal index (node - ntip) in its tree
};

struct Trees {
    u32 ntip, nbin, nnode1;
    const u32* par1;       // reference tree parent (0-based), n1 entries
    const u32* clade1;     // reference clade rows, (nnode1 - 1) x nbin, row k = node ntip + nnode1 - 1 - k
    const u64* nodeBase;   // per query tree: first internal node in the concatenated arrays
    const u32* kidOff;     // per tree (nnode + 1) absolute offsets into kid, at nodeBase[t] + t
    const u32* kid;        // children in edge order
    const u32* size;       // clade sizes of internal nodes
    const u32* rank;       // visiting rank of internal nodes (reverse edge order)
    u32* stop;             // stop node of internal nodes
    u32* rows;             // clade rows of internal nodes, nbin words each
    int32_t* q2r;          // qry2ref rows (node, distance, size)
    unsigned long long* key;  // per query tree, nnode1 keys
    float threshold;
};

__device__ __forceinline__ u32 stop_of(const Trees& T, u64 nb, u32 c) {
    return c < T.ntip ? __ldg(T.par1 + c) : T.stop[nb + (c - T.ntip)];
}

// One warp per internal node of one height: its clade row, then its walks.
__global__ void __launch_bounds__(kThreads) k_search(Trees T, const Item* __restrict__ items, u32 cnt) {
    const u32 w = (blockIdx.x * kThreads + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= cnt) return;
    const Item it = items[w];
    const u64 nb = T.nodeBase[it.tree];
    const u32* ko = T.kidOff + nb + it.tree;
    const u32 k0 = ko[it.node], k1 = ko[it.node + 1];
    const u32 nbin = T.nbin, ntip = T.ntip;
    u32* row = T.rows + (nb + it.node) * nbin;
    for (u32 x = lane; x < nbin; x += 32) {
        u32 acc = 0;
        for (u32 k = k0; k < k1; k++) {
            const u32 c = T.kid[k];
            if (c < ntip) acc |= (c >> 5) == x ? 1u << (c & 31) : 0u;
            else acc |= T.rows[(nb + (c - ntip)) * nbin + x];
        }
        row[x] = acc;
    }
    __syncwarp();
    const u32 size = T.size[nb + it.node];
    const float lim = __fmul_rn(__uint2float_rn(size), T.threshold);
    const u64 lowRank = (u64)(0xFFFFFFFFu - T.rank[nb + it.node]);
    unsigned long long* key = T.key + (u64)it.tree * T.nnode1;
    u32 stopd = stop_of(T, nb, T.kid[k0]);
    u32 best = 2u * ntip, m2 = 0u;
    for (u32 k = k0; k < k1; k++) {
        u32 cur = stop_of(T, nb, T.kid[k]);
        u32 nl = 0;
        while (cur > ntip && __uint2float_rn(nl) <= lim) {
            const u32 next = __ldg(T.par1 + cur);
            const u32 t1 = T.nnode1 - 1u - (cur - ntip);
            const u32* r1 = T.clade1 + (u64)t1 * nbin;
            u32 xr = 0;
            nl = 0;
            for (u32 x = lane; x < nbin; x += 32) {
                const u32 a = __ldg(r1 + x), b = row[x];
                xr += __popc(a ^ b);
                nl += __popc(a & ~b);
            }
            xr = __reduce_add_sync(0xFFFFFFFFu, xr);
            nl = __reduce_add_sync(0xFFFFFFFFu, nl);
            if (lane == 0) atomicMin(key + t1, (unsigned long long)(((u64)xr << 32) | lowRank));
            if (best >= xr) {
                best = xr;
                stopd = cur;
                m2 = cur + 1u;
            }
            cur = next;
        }
    }
    if (lane == 0) {
        T.stop[nb + it.node] = stopd;
        int32_t* q = T.q2r + (nb + it.node) * 3;
        q[0] = (int32_t)m2;
        q[1] = (int32_t)best;
        q[2] = (int32_t)size;
    }
}

// Per query tree: the qry2ref rows before the search (root (ntip+1, 0),
// others (0, 2 ntip), with the clade size; zero rows for a tree beyond the
// cache) and the node of each visiting rank.
__global__ void k_tree_init(u32 ntip, const u64* __restrict__ nodeBase, const u32* __restrict__ size,
                            const u32* __restrict__ rank, const u32* __restrict__ ok, const u32* __restrict__ roots,
                            u32* __restrict__ rankNode, int32_t* __restrict__ q2r) {
    const u32 t = blockIdx.x;
    const u64 nb = nodeBase[t], nn = nodeBase[t + 1] - nb;
    const bool good = ok[t] != 0;
    const u32 root = roots[t];
    for (u64 i = threadIdx.x; i < nn; i += blockDim.x) {
        int32_t* q = q2r + (nb + i) * 3;
        const u32 sz = size[nb + i];
        if (!good) {
            q[0] = q[1] = q[2] = 0;
        } else if (i == root) {
            q[0] = (int32_t)ntip + 1;
            q[1] = 0;
            q[2] = (int32_t)sz;
        } else {
            q[0] = 0;
            q[1] = (int32_t)(2u * ntip);
            q[2] = (int32_t)sz;
            rankNode[nb + rank[nb + i]] = (u32)i;
        }
    }
}

// ref2qry rows of every query tree from the keys: row 0 the root (ntip+1, 0),
// row i the reference node ntip+i; untouched nodes keep (0, 2 ntip).
__global__ void k_ref2qry(u32 ntree, u32 nnode1, u32 ntip, const unsigned long long* __restrict__ key,
                          const u64* __restrict__ nodeBase, const u32* __restrict__ rankNode,
                          const u32* __restrict__ treeOk, int32_t* __restrict__ out) {
    const u64 id = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= (u64)ntree * nnode1) return;
    const u32 t = (u32)(id / nnode1), i = (u32)(id % nnode1);
    int32_t* o = out + id * 2;
    if (!treeOk[t]) {
        o[0] = 0;
        o[1] = 0;
        return;
    }
    if (i == 0) {
        o[0] = (int32_t)ntip + 1;
        o[1] = 0;
        return;
    }
    const unsigned long long k = key[(u64)t * nnode1 + (nnode1 - 1u - i)];
    if (k == ~0ull) {
        o[0] = 0;
        o[1] = (int32_t)(2u * ntip);
    } else {
        const u32 rank = 0xFFFFFFFFu - (u32)(k & 0xFFFFFFFFull);
        o[0] = (int32_t)(rankNode[nodeBase[t] + rank] + ntip + 1u);
        o[1] = (int32_t)(k >> 32);
    }
}

// cal.abs: per reference node, the fraction of query trees whose best XOR
// distance divided by the node's size (binary64) is at most the threshold.
__global__ void k_support(u32 ntree, u32 nnode1, u32 ntip, const unsigned long long* __restrict__ key,
                          const int32_t* __restrict__ nodeSize, double threshold, double* __restrict__ support) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nnode1) return;
    const double sz = (double)nodeSize[i];
    u32 n = 0;
    for (u32 t = 0; t < ntree; t++) {
        u32 dis = 0;
        if (i > 0) {
            const unsigned long long k = key[(u64)t * nnode1 + (nnode1 - 1u - i)];
            dis = k == ~0ull ? 2u * ntip : (u32)(k >> 32);
        }
        n += __ddiv_rn((double)dis, sz) <= threshold;
    }
    support[i] = __ddiv_rn((double)n, (double)ntree);
}

// nodeDesBig rows of the reference tree, one height at a time (row of node v
// at rowOf[v - ntip]; the root's row is the extra last one).
__global__ void k_clade_rows(u32 ntip, u32 nbin, const u32* __restrict__ order, u32 off, u32 cnt,
                             const u32* __restrict__ kidOff, const u32* __restrict__ kid, const u32* __restrict__ rowOf,
                             u32* rows) {
    const u64 id = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= (u64)cnt * nbin) return;
    const u32 i = order[off + (u32)(id / nbin)], x = (u32)(id % nbin);
    u32 acc = 0;
    for (u32 k = kidOff[i]; k < kidOff[i + 1]; k++) {
        const u32 c = kid[k];
        if (c < ntip) acc |= (c >> 5) == x ? 1u << (c & 31) : 0u;
        else acc |= rows[(u64)rowOf[c - ntip] * nbin + x];
    }
    rows[(u64)rowOf[i] * nbin + x] = acc;
}

}  // namespace tsup

namespace {

inline u32 nblocks(u64 n, u32 t) { return (u32)((n + t - 1) / t); }

// f(i) for i < n on up to 32 host threads (the per-tree host work).
template <class F>
void parallel_for(u32 n, F f) {
    const u32 hw = std::max(1u, std::thread::hardware_concurrency());
    const u32 nt = std::min(n, std::min(hw, 32u));
    if (nt <= 1) {
        for (u32 i = 0; i < n; i++) f(i);
        return;
    }
    std::atomic<u32> next{0};
    std::vector<std::thread> th;
    th.reserve(nt);
    for (u32 k = 0; k < nt; k++)
        th.emplace_back([&] {
            for (u32 i; (i = next.fetch_add(1)) < n;) f(i);
        });
    for (auto& t : th) t.join();
}

// One rooted tree as the reference's loops see it: children in edge order,
// heights, sizes, the reverse-edge visiting rank of internal children and
// whether the 8192-row cache suffices.
struct QTree {
    u32 nnode = 0, root = 0, height = 0;
    bool cacheOk = true;
    std::vector<u32> kidOff, kid, size, rank, rankNode, h;
};

int parse_tree(u32 ntip, u32 nedge, const u32* edge, u32 cacheSize, QTree& Q, const char* who) {
    if (nedge < ntip || !edge) {
        casphy_set_last_error_msg(who);
        return CASPHY_EINVAL;
    }
    const u32 nnode = nedge - ntip + 1, nn = ntip + nnode, none = 0xFFFFFFFFu;
    Q.nnode = nnode;
    std::vector<u32> pe(nn, none);
    Q.kidOff.assign(nnode + 1, 0);
    for (u32 e = 0; e < nedge; e++) {
        const u32 a = edge[2 * e], d = edge[2 * e + 1];
        if (a < ntip || a >= nn || d >= nn || a == d || pe[d] != none) {
            casphy_set_last_error_msg(who);
            return CASPHY_EINVAL;
        }
        pe[d] = e;
        Q.kidOff[a - ntip + 1]++;
    }
    u32 nroot = 0;
    for (u32 v = 0; v < nn; v++)
        if (pe[v] == none) {
            if (v < ntip) nroot = 2;
            Q.root = v;
            nroot++;
        }
    if (nroot != 1) {
        casphy_set_last_error_msg(who);
        return CASPHY_EINVAL;
    }
    for (u32 e = 0; e < nedge; e++) {
        const u32 a = edge[2 * e];
        if (a != Q.root && pe[a] > e) {  // the edge into a node comes before its own edges
            casphy_set_last_error_msg(who);
            return CASPHY_EINVAL;
        }
    }
    for (u32 i = 0; i < nnode; i++) {
        if (Q.kidOff[i + 1] == 0) {
            casphy_set_last_error_msg(who);
            return CASPHY_EINVAL;
        }
        Q.kidOff[i + 1] += Q.kidOff[i];
    }
    Q.kid.assign(nedge, 0);
    std::vector<u32> fill(Q.kidOff.begin(), Q.kidOff.end() - 1);
    for (u32 e = 0; e < nedge; e++) Q.kid[fill[edge[2 * e] - ntip]++] = edge[2 * e + 1];
    Q.size.assign(nnode, 0);
    Q.rank.assign(nnode, 0);
    Q.rankNode.assign(nnode, 0);
    Q.h.assign(nnode, 0);
    std::vector<unsigned char> open(nnode, 0);
    u32 nUse = 0, r = 0;
    for (u32 e = nedge; e-- > 0;) {
        const u32 a = edge[2 * e] - ntip, d = edge[2 * e + 1];
        if (!open[a]) {
            if (nUse == cacheSize) Q.cacheOk = false;
            open[a] = 1;
            nUse++;
        }
        if (d < ntip) {
            Q.size[a]++;
            Q.h[a] = std::max(Q.h[a], 1u);
        } else {
            const u32 di = d - ntip;
            Q.size[a] += Q.size[di];
            Q.h[a] = std::max(Q.h[a], Q.h[di] + 1);
            Q.rank[di] = r;
            Q.rankNode[r] = di;
            r++;
            open[di] = 0;
            nUse--;
        }
    }
    Q.height = Q.h[Q.root - ntip];
    return CASPHY_OK;
}

}  // namespace
}  // namespace casphy

namespace casphy {
namespace {

using tsup::Item;

constexpr u64 kRowBudget = 8ull << 30;  // clade rows of the query trees held at once

// Parents of the reference tree (0-based, root ntip).
int parents(u32 ntip, u32 nedge, const u32* edge, std::vector<u32>& par, u32& nnode) {
    if (!edge || nedge < ntip) return CASPHY_EINVAL;
    nnode = nedge - ntip + 1;
    const u32 nn = ntip + nnode;
    par.assign(nn, 0xFFFFFFFFu);
    for (u32 e = 0; e < nedge; e++) {
        const u32 a = edge[2 * e], d = edge[2 * e + 1];
        if (a < ntip || a >= nn || d >= nn || a == d || par[d] != 0xFFFFFFFFu) return CASPHY_EINVAL;
        par[d] = a;
    }
    for (u32 v = 0; v < nn; v++)
        if ((par[v] == 0xFFFFFFFFu) != (v == ntip)) return CASPHY_EINVAL;
    // every node reaches the root
    std::vector<unsigned char> seen(nn, 0);
    seen[ntip] = 2;
    for (u32 v = 0; v < nn; v++) {
        u32 u = v, steps = 0;
        while (!seen[u]) {
            seen[u] = 1;
            u = par[u];
            if (++steps > nn) return CASPHY_EINVAL;
        }
        if (seen[u] == 1) return CASPHY_EINVAL;  // back on this path: a cycle
        for (u32 w = v; seen[w] == 1; w = par[w]) seen[w] = 2;
    }
    return CASPHY_OK;
}

struct Group {
    u32 t0, t1;  // query trees [t0, t1)
    u64 nNode, nKid, nItem;
};

// The whole comparison for one reference tree.  Reference tree: parents par1
// and either its clade rows (rowsHost, nodeDesBig order) or its parsed tree
// (Q1, rows computed here).  Outputs (each optional): ref2qry rows of every
// query tree, qry2ref rows concatenated, cal.abs support with node sizes.
int compare_all(u32 ntip, u32 nnode1, const std::vector<u32>& par1, const u32* rowsHost, const QTree* Q1,
                const std::vector<QTree>& Q, float threshold, int32_t* ref2qry, int32_t* qry2ref,
                const int32_t* nodeSizeHost, double supThr, double* support) {
    using namespace tsup;
    const u32 nbin = ((ntip - 1) >> 5) + 1, ntree = (u32)Q.size(), n1 = ntip + nnode1;
    // groups of query trees whose clade rows fit the budget
    std::vector<Group> groups;
    {
        Group g{0, 0, 0, 0, 0};
        for (u32 t = 0; t < ntree; t++) {
            const u64 nn = Q[t].nnode, nk = Q[t].kid.size();
            if (g.t1 > g.t0 && (g.nNode + nn) * nbin * 4 > kRowBudget) {
                groups.push_back(g);
                g = Group{t, t, 0, 0, 0};
            }
            g.t1 = t + 1;
            g.nNode += nn;
            g.nKid += nk;
            if (Q[t].cacheOk) g.nItem += nn - 1;
        }
        if (g.t1 > g.t0) groups.push_back(g);
    }
    u64 mxNode = 1, mxKid = 1, mxItem = 1, mxTree = 1;
    for (const Group& g : groups) {
        mxNode = std::max(mxNode, g.nNode);
        mxKid = std::max(mxKid, g.nKid);
        mxItem = std::max(mxItem, g.nItem);
        mxTree = std::max<u64>(mxTree, g.t1 - g.t0);
    }
    struct Lay {
        u32 *par1, *clade1, *kidOff1, *kid1, *rowOf1, *order1;
        unsigned long long* key;
        int32_t *r2q, *nodeSize;
        double* support;
        u64* nodeBase;
        u32 *kidOff, *kid, *size, *rank, *rankNode, *stop, *rows, *ok, *roots;
        int32_t* q2r;
        Item* items;
    };
    const u32 nkid1 = Q1 ? (u32)Q1->kid.size() : 1u;
    auto lay = [&](Carve& c) {
        Lay l;
        l.par1 = c.take<u32>(n1);
        l.clade1 = c.take<u32>((u64)nnode1 * nbin);
        l.kidOff1 = c.take<u32>(Q1 ? nnode1 + 1 : 1);
        l.kid1 = c.take<u32>(nkid1);
        l.rowOf1 = c.take<u32>(Q1 ? nnode1 : 1);
        l.order1 = c.take<u32>(Q1 ? nnode1 : 1);
        l.key = c.take<unsigned long long>((u64)ntree * nnode1);
        l.r2q = c.take<int32_t>(ref2qry ? (u64)ntree * nnode1 * 2 : 1);
        l.nodeSize = c.take<int32_t>(nnode1);
        l.support = c.take<double>(nnode1);
        l.nodeBase = c.take<u64>(mxTree + 1);
        l.kidOff = c.take<u32>(mxNode + mxTree);
        l.kid = c.take<u32>(mxKid);
        l.size = c.take<u32>(mxNode);
        l.rank = c.take<u32>(mxNode);
        l.rankNode = c.take<u32>(mxNode);
        l.stop = c.take<u32>(mxNode);
        l.rows = c.take<u32>(mxNode * nbin);
        l.ok = c.take<u32>(mxTree);
        l.roots = c.take<u32>(mxTree);
        l.q2r = c.take<int32_t>(mxNode * 3);
        l.items = c.take<Item>(mxItem);
        return l;
    };
    Carve cv;
    lay(cv);
    DeviceScope ds;
    void* base = nullptr;
    int rc = ds.reserve(cv.off + 256, &base);
    if (rc) return rc;
    Carve c2;
    c2.base = static_cast<char*>(base);
    const Lay L = lay(c2);
    cudaStream_t st = 0;
    CASPHY_CUDA_TRY(cudaMemcpyAsync(L.par1, par1.data(), 4ull * n1, cudaMemcpyHostToDevice, st));
    if (rowsHost) {
        if (nnode1 > 1)
            CASPHY_CUDA_TRY(cudaMemcpyAsync(L.clade1, rowsHost, 4ull * (nnode1 - 1) * nbin, cudaMemcpyHostToDevice, st));
    } else {
        // nodeDesBig rows of the reference tree: node i at its closing rank,
        // the root at the extra last row; one launch per height
        const QTree& q = *Q1;
        std::vector<u32> rowOf(nnode1), order;
        std::vector<u32> hOff(q.height + 2, 0);
        for (u32 i = 0; i < nnode1; i++) {
            rowOf[i] = i == q.root - ntip ? nnode1 - 1 : q.rank[i];
            hOff[q.h[i] + 1]++;
        }
        for (u32 l = 1; l <= q.height + 1; l++) hOff[l] += hOff[l - 1];
        order.resize(nnode1);
        {
            std::vector<u32> pos(hOff.begin(), hOff.end() - 1);
            for (u32 i = 0; i < nnode1; i++) order[pos[q.h[i]]++] = i;
        }
        CASPHY_CUDA_TRY(cudaMemcpyAsync(L.kidOff1, q.kidOff.data(), 4ull * (nnode1 + 1), cudaMemcpyHostToDevice, st));
        CASPHY_CUDA_TRY(cudaMemcpyAsync(L.kid1, q.kid.data(), 4ull * q.kid.size(), cudaMemcpyHostToDevice, st));
        CASPHY_CUDA_TRY(cudaMemcpyAsync(L.rowOf1, rowOf.data(), 4ull * nnode1, cudaMemcpyHostToDevice, st));
        CASPHY_CUDA_TRY(cudaMemcpyAsync(L.order1, order.data(), 4ull * nnode1, cudaMemcpyHostToDevice, st));
        for (u32 l = 1; l <= q.height; l++) {
            const u32 cnt = hOff[l + 1] - hOff[l];
            if (cnt)
                k_clade_rows<<<nblocks((u64)cnt * nbin, 256), 256, 0, st>>>(ntip, nbin, L.order1, hOff[l], cnt,
                                                                          L.kidOff1, L.kid1, L.rowOf1, L.clade1);
        }
        CASPHY_CUDA_TRY(cudaGetLastError());
    }
    CASPHY_CUDA_TRY(cudaMemsetAsync(L.key, 0xFF, 8ull * ntree * nnode1, st));
    u64 qOut = 0;  // qry2ref rows written so far
    for (const Group& g : groups) {
        const u32 nt = g.t1 - g.t0;
        std::vector<u64> nodeBase(nt + 1, 0), kidBase(nt + 1, 0);
        std::vector<u32> ok(nt), roots(nt);
        u32 H = 0;
        for (u32 t = 0; t < nt; t++) {
            const QTree& q = Q[g.t0 + t];
            nodeBase[t + 1] = nodeBase[t] + q.nnode;
            kidBase[t + 1] = kidBase[t] + q.kid.size();
            ok[t] = q.cacheOk;
            roots[t] = q.root - ntip;
            if (q.cacheOk) H = std::max(H, q.height);
        }
        const u64 nNode = nodeBase[nt];
        if (kidBase[nt] > 0xFFFFFFFFull) return CASPHY_ERANGE;
        // the searched nodes (internal, not the root) counted per tree and
        // height, then placed height by height
        const u64 nh = (u64)H + 1;
        std::vector<u64> cnt((u64)nt * nh, 0), pos((u64)nt * nh, 0), lvlOff(nh + 1, 0);
        parallel_for(nt, [&](u32 t) {
            const QTree& q = Q[g.t0 + t];
            if (!q.cacheOk) return;
            u64* c = cnt.data() + t * nh;
            for (u32 i = 0; i < q.nnode; i++)
                if (i != q.root - ntip) c[q.h[i]]++;
        });
        {
            u64 o = 0;
            for (u64 l = 0; l < nh; l++) {
                lvlOff[l] = o;
                for (u32 t = 0; t < nt; t++) {
                    pos[t * nh + l] = o;
                    o += cnt[t * nh + l];
                }
            }
            lvlOff[nh] = o;
        }
        std::vector<u32> kidOff(nNode + nt), kid(std::max<u64>(kidBase[nt], 1)), size(nNode), rank(nNode);
        std::vector<Item> items(std::max<u64>(lvlOff[nh], 1));
        parallel_for(nt, [&](u32 t) {
            const QTree& q = Q[g.t0 + t];
            const u64 nb = nodeBase[t], kb = kidBase[t];
            for (u32 i = 0; i <= q.nnode; i++) kidOff[nb + t + i] = (u32)(kb + q.kidOff[i]);
            std::copy(q.kid.begin(), q.kid.end(), kid.begin() + kb);
            std::copy(q.size.begin(), q.size.end(), size.begin() + nb);
            std::copy(q.rank.begin(), q.rank.end(), rank.begin() + nb);
            if (!q.cacheOk) return;
            u64* p = pos.data() + t * nh;
            for (u32 i = 0; i < q.nnode; i++)
                if (i != q.root - ntip) items[p[q.h[i]]++] = Item{t, i};
        });
        CASPHY_CUDA_TRY(cudaMemcpyAsync(L.nodeBase, nodeBase.data(), 8ull * (nt + 1), cudaMemcpyHostToDevice, st));
        CASPHY_CUDA_TRY(cudaMemcpyAsync(L.kidOff, kidOff.data(), 4ull * kidOff.size(), cudaMemcpyHostToDevice, st));
        CASPHY_CUDA_TRY(cudaMemcpyAsync(L.kid, kid.data(), 4ull * kid.size(), cudaMemcpyHostToDevice, st));
        CASPHY_CUDA_TRY(cudaMemcpyAsync(L.size, size.data(), 4ull * nNode, cudaMemcpyHostToDevice, st));
        CASPHY_CUDA_TRY(cudaMemcpyAsync(L.rank, rank.data(), 4ull * nNode, cudaMemcpyHostToDevice, st));
        CASPHY_CUDA_TRY(cudaMemcpyAsync(L.ok, ok.data(), 4ull * nt, cudaMemcpyHostToDevice, st));
        CASPHY_CUDA_TRY(cudaMemcpyAsync(L.roots, roots.data(), 4ull * nt, cudaMemcpyHostToDevice, st));
        CASPHY_CUDA_TRY(cudaMemcpyAsync(L.items, items.data(), sizeof(Item) * items.size(), cudaMemcpyHostToDevice, st));
        k_tree_init<<<nt, 256, 0, st>>>(ntip, L.nodeBase, L.size, L.rank, L.ok, L.roots, L.rankNode, L.q2r);
        const u32 H1 = H;
        Trees T;
        T.ntip = ntip;
        T.nbin = nbin;
        T.nnode1 = nnode1;
        T.par1 = L.par1;
        T.clade1 = L.clade1;
        T.nodeBase = L.nodeBase;
        T.kidOff = L.kidOff;
        T.kid = L.kid;
        T.size = L.size;
        T.rank = L.rank;
        T.stop = L.stop;
        T.rows = L.rows;
        T.q2r = L.q2r;
        T.key = L.key + (u64)g.t0 * nnode1;
        T.threshold = threshold;
        for (u32 l = 1; l <= H1; l++) {
            const u64 c = lvlOff[l + 1] - lvlOff[l];
            if (c) k_search<<<nblocks(c * 32, kThreads), kThreads, 0, st>>>(T, L.items + lvlOff[l], (u32)c);
        }
        CASPHY_CUDA_TRY(cudaGetLastError());
        if (ref2qry)
            k_ref2qry<<<nblocks((u64)nt * nnode1, 256), 256, 0, st>>>(nt, nnode1, ntip, T.key, L.nodeBase, L.rankNode,
                                                                     L.ok, L.r2q + (u64)g.t0 * nnode1 * 2);
        CASPHY_CUDA_TRY(cudaGetLastError());
        if (qry2ref)
            CASPHY_CUDA_TRY(cudaMemcpyAsync(qry2ref + qOut * 3, L.q2r, 12ull * nNode, cudaMemcpyDeviceToHost, st));
        CASPHY_CUDA_TRY(cudaStreamSynchronize(st));
        qOut += nNode;
    }
    if (ref2qry)
        CASPHY_CUDA_TRY(cudaMemcpyAsync(ref2qry, L.r2q, 8ull * ntree * nnode1, cudaMemcpyDeviceToHost, st));
    if (support) {
        CASPHY_CUDA_TRY(cudaMemcpyAsync(L.nodeSize, nodeSizeHost, 4ull * nnode1, cudaMemcpyHostToDevice, st));
        tsup::k_support<<<nblocks(nnode1, 256), 256, 0, st>>>(ntree, nnode1, ntip, L.key, L.nodeSize, supThr,
                                                             L.support);
        CASPHY_CUDA_TRY(cudaGetLastError());
        CASPHY_CUDA_TRY(cudaMemcpyAsync(support, L.support, 8ull * nnode1, cudaMemcpyDeviceToHost, st));
    }
    CASPHY_CUDA_TRY(cudaStreamSynchronize(st));
    return CASPHY_OK;
}

int parse_queries(u32 ntip, u32 ntree, const uint64_t* edge_off, const uint32_t* edges2, u32 cacheSize,
                  std::vector<QTree>& Q) {
    if (!edge_off || !edges2) return CASPHY_EINVAL;
    for (u32 t = 0; t < ntree; t++)
        if (edge_off[t + 1] < edge_off[t] || edge_off[t + 1] - edge_off[t] > 0xFFFFFFFFull) return CASPHY_EINVAL;
    static const char* kMsg =
        "approximateCompare: each query tree must be one rooted tree, edges in cladewise order (a node's parent "
        "edge before its own edges)";
    Q.resize(ntree);
    std::vector<int> rcs(ntree, 0);
    parallel_for(ntree, [&](u32 t) {
        rcs[t] = parse_tree(ntip, (u32)(edge_off[t + 1] - edge_off[t]), edges2 + 2 * edge_off[t], cacheSize, Q[t],
                            kMsg);
    });
    for (u32 t = 0; t < ntree; t++)
        if (rcs[t]) {
            casphy_set_last_error_msg(kMsg);  // the workers' messages stay on their threads
            return rcs[t];
        }
    return CASPHY_OK;
}

}  // namespace
}  // namespace casphy

extern "C" int casphy_approx_compare(uint32_t ntip, uint32_t nnode1, const uint32_t* clade_rows, uint32_t nedge1,
                                     const uint32_t* edge1, uint32_t ntree, const uint64_t* edge_off,
                                     const uint32_t* edges2, uint32_t cache_size, float threshold, int32_t* ref2qry,
                                     int32_t* qry2ref, int32_t* status) {
    using namespace casphy;
    int rc = require_device();
    if (rc) return rc;
    if (ntip < 2 || !clade_rows || !status || (ntree && (!ref2qry || !qry2ref)) || !(threshold == threshold))
        return CASPHY_EINVAL;
    std::vector<u32> par1;
    u32 nn1 = 0;
    if (parents(ntip, nedge1, edge1, par1, nn1) || nn1 != nnode1) {
        casphy_set_last_error_msg("approximateCompare: the reference tree must be one rooted tree with root ntip");
        return CASPHY_EINVAL;
    }
    std::vector<QTree> Q;
    if ((rc = parse_queries(ntip, ntree, edge_off, edges2, cache_size, Q))) return rc;
    for (u32 t = 0; t < ntree; t++) status[t] = Q[t].cacheOk ? CASPHY_OK : CASPHY_ERANGE;
    if (!ntree) return CASPHY_OK;
    return compare_all(ntip, nnode1, par1, clade_rows, nullptr, Q, threshold, ref2qry, qry2ref, nullptr, 0.0,
                       nullptr);
}

extern "C" int casphy_cal_abs(uint32_t ntip, uint32_t nedge1, const uint32_t* edge1, uint32_t ntree,
                              const uint64_t* edge_off, const uint32_t* edges2, double threshold, double* support,
                              int32_t* node_size) {
    using namespace casphy;
    int rc = require_device();
    if (rc) return rc;
    if (ntip < 2 || ntree == 0 || !support || !node_size || !(threshold == threshold)) return CASPHY_EINVAL;
    std::vector<u32> par1;
    u32 nnode1 = 0;
    if (parents(ntip, nedge1, edge1, par1, nnode1)) {
        casphy_set_last_error_msg("cal.abs: the reference tree must be one rooted tree with root ntip");
        return CASPHY_EINVAL;
    }
    QTree Q1;
    if ((rc = parse_tree(ntip, nedge1, edge1, 8192, Q1,
                         "cal.abs: reference tree edges must be in cladewise order")))
        return rc;
    if (!Q1.cacheOk) {
        casphy_set_last_error_msg("Run out of cache!");
        return CASPHY_ERANGE;
    }
    std::vector<QTree> Q;
    if ((rc = parse_queries(ntip, ntree, edge_off, edges2, 8192, Q))) return rc;
    for (u32 t = 0; t < ntree; t++)
        if (!Q[t].cacheOk) {
            casphy_set_last_error_msg("Run out of cache!");
            return CASPHY_ERANGE;
        }
    // phy2clade's node sizes: ntip for the root, then the internal nodes in order
    node_size[0] = (int32_t)ntip;
    for (u32 i = 1; i < nnode1; i++) node_size[i] = (int32_t)Q1.size[i];
    // R passes threshold + 0.05 (binary64) to the binary32 parameter
    const float cmpThr = (float)(threshold + 0.05);
    return compare_all(ntip, nnode1, par1, nullptr, &Q1, Q, cmpThr, nullptr, nullptr, node_size, threshold, support);
}
