// Tree passes of the reference's CPU helpers on B200: parsimony change counts
// per edge, the reference's branch-length surrogate (ancestralBitReverse and
// charAncestralEC, src/functions.cpp:3478-3542 and 3085-3150, called by
// collapse.infoless / cal.nevo, R/CasPhy_functions.R:804-845), and the clade
// rows of nodeDesBig (src/functions.cpp:1277-1366), the TransferDisStream
// input that phy2clade writes (R/bootstrap_functions.R:1-32).
//
// Both are a bottom-up pass followed by a per-edge count.  The reference runs
// the bottom-up pass over the edge rows in reverse order, so for every
// internal node the children are folded in reverse edge order and every
// child is complete before its parent; here the internal nodes are grouped by
// height and one launch folds one height level, one thread per (node, word)
// or (node, site), children in the same reverse edge order (the fold is
// order-dependent at multifurcations).  The bit version then resolves the
// bistate bits of every internal child from its parent in pre-order (one
// launch per depth level) and counts the changed bits per edge; the indel
// version counts the sites where both ends are known and differ.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "runtime.h"

namespace casphy {
namespace pars {

struct Tree {
    u32 ntip;
    const u32* kidOff;   // internal node i = v - ntip: children kid[kidOff[i] .. kidOff[i+1])
    const u32* kid;      // child node id, in edge order
    const u32* kidEdge;  // the edge row of that child
    const u32* order;    // internal nodes, grouped by level
};

// bottom-up fold, bit version: state = AND of children, bistate = AND of
// children's bistates (tips 0), conflict = differing, non-bistate bits; a
// child's conflict bits join its state and bistate as it is folded
__global__ void k_up_bit(Tree T, u32 off, u32 cnt, u32 nbin, const u32* __restrict__ mat, u32* state, u32* bis,
                         u32* conf) {
    const u64 id = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= (u64)cnt * nbin) return;
    const u32 i = T.order[off + (u32)(id / nbin)] - T.ntip, w = (u32)(id % nbin);
    u32 s1 = 0xFFFFFFFFu, b1 = 0xFFFFFFFFu, cf = 0;
    for (u32 k = T.kidOff[i + 1]; k-- > T.kidOff[i];) {
        const u32 d = T.kid[k];
        u32 s2, b2;
        if (d < T.ntip) {
            s2 = mat[(size_t)d * nbin + w];
            b2 = 0;
        } else {
            const size_t j = (size_t)(d - T.ntip) * nbin + w;
            const u32 c = conf[j];
            s2 = state[j] | c;
            b2 = bis[j] | c;
            state[j] = s2;
            bis[j] = b2;
        }
        cf |= (s1 ^ s2) & ~(b1 | b2);
        s1 &= s2;
        b1 &= b2;
    }
    const size_t j = (size_t)i * nbin + w;
    state[j] = s1;
    bis[j] = b1;
    conf[j] = cf;
}

__global__ void k_root_bit(u32 nbin, u32* state, const u32* bis, const u32* conf) {
    const u32 w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w < nbin) state[w] &= ~(conf[w] | bis[w]);
}

// top-down, bit version: every child of a node at this depth level takes its
// parent's bits where it is bistate; changed bits are counted per edge
__global__ void k_down_bit(Tree T, u32 off, u32 cnt, u32 nbin, const u32* __restrict__ mat, u32* state,
                           const u32* __restrict__ bis, u32* len) {
    const u64 id = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= (u64)cnt * nbin) return;
    const u32 i = T.order[off + (u32)(id / nbin)] - T.ntip, w = (u32)(id % nbin);
    const u32 sa = state[(size_t)i * nbin + w];
    for (u32 k = T.kidOff[i]; k < T.kidOff[i + 1]; k++) {
        const u32 d = T.kid[k];
        u32 n;
        if (d < T.ntip) {
            n = __popc(sa ^ mat[(size_t)d * nbin + w]);
        } else {
            const size_t j = (size_t)(d - T.ntip) * nbin + w;
            const u32 bd = bis[j];
            const u32 t = (state[j] & ~bd) | (sa & bd);
            state[j] = t;
            n = __popc(sa ^ t);
        }
        if (n) atomicAdd(len + T.kidEdge[k], n);
    }
}

// bottom-up fold, indel version: the first known child value of each site,
// 0 where a later known child disagrees; children failing the size rule are
// skipped (use[edge] == 0)
__global__ void k_up_char(Tree T, u32 off, u32 cnt, u32 nsite, const int* __restrict__ mat,
                          const unsigned char* __restrict__ use, int* state) {
    const u64 id = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= (u64)cnt * nsite) return;
    const u32 i = T.order[off + (u32)(id / nsite)] - T.ntip, s = (u32)(id % nsite);
    int cur = -1;
    for (u32 k = T.kidOff[i + 1]; k-- > T.kidOff[i];) {
        if (!use[T.kidEdge[k]]) continue;
        const u32 d = T.kid[k];
        const int v = d < T.ntip ? mat[(size_t)d * nsite + s] : state[(size_t)(d - T.ntip) * nsite + s];
        if (cur == -1) cur = v;
        else if (cur != v && v != -1) cur = 0;
    }
    state[(size_t)i * nsite + s] = cur;
}

// edge lengths, indel version: one block per edge
__global__ void k_len_char(u32 ntip, u32 nedge, u32 nsite, const u32* __restrict__ edge, const int* __restrict__ mat,
                           const int* __restrict__ state, u32* len) {
    __shared__ u32 red[32];
    const u32 e = blockIdx.x;
    if (e >= nedge) return;
    const u32 a = edge[2 * e], d = edge[2 * e + 1];
    const int* pa = state + (size_t)(a - ntip) * nsite;
    const int* pd = d < ntip ? mat + (size_t)d * nsite : state + (size_t)(d - ntip) * nsite;
    u32 n = 0;
    for (u32 s = threadIdx.x; s < nsite; s += blockDim.x) {
        const int x = pa[s], y = pd[s];
        n += x >= 0 && y >= 0 && x != y;
    }
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xFFFFFFFFu, n, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = n;
    __syncthreads();
    if (threadIdx.x == 0) {
        u32 t = 0;
        for (u32 k = 0; k < blockDim.x / 32; k++) t += red[k];
        len[e] = t;
    }
}

// clade rows, one height level: thread per (node, word); a node's row is the
// OR of its tip children's bits and its internal children's rows; rows live
// at their output positions (rowOf), the root in the extra last row
__global__ void k_clade(Tree T, u32 off, u32 cnt, u32 nbin, const u32* __restrict__ rowOf, u32* rows) {
    const u64 id = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= (u64)cnt * nbin) return;
    const u32 v = T.order[off + (u32)(id / nbin)], i = v - T.ntip, w = (u32)(id % nbin);
    u32 acc = 0;
    for (u32 k = T.kidOff[i]; k < T.kidOff[i + 1]; k++) {
        const u32 d = T.kid[k];
        if (d < T.ntip) acc |= (d >> 5) == w ? 1u << (d & 31) : 0u;
        else acc |= rows[(size_t)rowOf[d - T.ntip] * nbin + w];
    }
    rows[(size_t)rowOf[i] * nbin + w] = acc;
}

}  // namespace pars

using namespace pars;

namespace {

struct HostTree {
    u32 ntip = 0, nnode = 0, root = 0;
    std::vector<u32> kidOff, kid, kidEdge, upOrder, downOrder, upOff, downOff;
    std::vector<u32> parentEdge;
};

// Children in edge order, height and depth levels; the edge rows must list
// the edge into a node before the node's own edges (pre-order, as an ape
// cladewise edge matrix), which is what the reference's passes rely on.
int build(u32 ntip, u32 nnode, u32 nedge, const u32* edge, HostTree& T) {
    const u32 nn = ntip + nnode, none = 0xFFFFFFFFu;
    if (!edge || nnode == 0 || nedge == 0) return CASPHY_EINVAL;
    T.ntip = ntip;
    T.nnode = nnode;
    T.parentEdge.assign(nn, none);
    std::vector<u32> nk(nnode + 1, 0);
    for (u32 e = 0; e < nedge; e++) {
        const u32 a = edge[2 * e], d = edge[2 * e + 1];
        if (a < ntip || a >= nn || d >= nn || a == d || T.parentEdge[d] != none) {
            casphy_set_last_error_msg("parsimony: bad edge (parents must be internal, one parent per node)");
            return CASPHY_EINVAL;
        }
        T.parentEdge[d] = e;
        nk[a - ntip + 1]++;
    }
    u32 nroot = 0;
    for (u32 v = ntip; v < nn; v++)
        if (T.parentEdge[v] == none) {
            T.root = v;
            nroot++;
        }
    for (u32 v = 0; v < ntip; v++)
        if (T.parentEdge[v] == none) {
            casphy_set_last_error_msg("parsimony: every tip needs a parent edge");
            return CASPHY_EINVAL;
        }
    if (nroot != 1) {
        casphy_set_last_error_msg("parsimony: the edges must form one rooted tree");
        return CASPHY_EINVAL;
    }
    for (u32 e = 0; e < nedge; e++) {
        const u32 a = edge[2 * e];
        if (a != T.root && T.parentEdge[a] > e) {
            casphy_set_last_error_msg("parsimony: edge rows must list a node's parent edge before its own edges");
            return CASPHY_EINVAL;
        }
    }
    for (u32 i = 0; i < nnode; i++) {
        if (nk[i + 1] == 0) {
            casphy_set_last_error_msg("parsimony: an internal node has no children");
            return CASPHY_EINVAL;
        }
        nk[i + 1] += nk[i];
    }
    T.kidOff = nk;
    T.kid.assign(nedge, 0);
    T.kidEdge.assign(nedge, 0);
    std::vector<u32> fill(nk.begin(), nk.end() - 1);
    for (u32 e = 0; e < nedge; e++) {
        const u32 a = edge[2 * e] - ntip;
        T.kid[fill[a]] = edge[2 * e + 1];
        T.kidEdge[fill[a]] = e;
        fill[a]++;
    }
    // depth in edge order (parents first), height in reverse edge order
    std::vector<u32> depth(nn, 0), height(nn, 0);
    for (u32 e = 0; e < nedge; e++) depth[edge[2 * e + 1]] = depth[edge[2 * e]] + 1;
    for (u32 e = nedge; e-- > 0;) {
        const u32 a = edge[2 * e], d = edge[2 * e + 1];
        height[a] = std::max(height[a], d < ntip ? 1u : height[d] + 1);
    }
    u32 H = 0, D = 0;
    for (u32 v = ntip; v < nn; v++) {
        H = std::max(H, height[v]);
        D = std::max(D, depth[v]);
    }
    std::vector<std::vector<u32>> byH(H + 1), byD(D + 1);
    for (u32 v = ntip; v < nn; v++) {
        byH[height[v]].push_back(v);
        byD[depth[v]].push_back(v);
    }
    T.upOff.assign(1, 0);
    for (u32 h = 1; h <= H; h++) {
        T.upOrder.insert(T.upOrder.end(), byH[h].begin(), byH[h].end());
        T.upOff.push_back((u32)T.upOrder.size());
    }
    T.downOff.assign(1, 0);
    for (u32 d = 0; d <= D; d++) {
        if (byD[d].empty()) continue;
        T.downOrder.insert(T.downOrder.end(), byD[d].begin(), byD[d].end());
        T.downOff.push_back((u32)T.downOrder.size());
    }
    return CASPHY_OK;
}

struct DevTree {
    u32 *kidOff, *kid, *kidEdge, *up, *down;
};

template <class B, class Lay>
int reserve_and_upload(DeviceScope& ds, const HostTree& H, Lay lay, B& L, DevTree& D, cudaStream_t st) {
    Carve cv;
    lay(cv);
    const u32 nedge = (u32)H.kid.size(), nnode = H.nnode;
    cv.take<u32>(nnode + 1);
    cv.take<u32>(nedge);
    cv.take<u32>(nedge);
    cv.take<u32>(nnode);
    cv.take<u32>(nnode);
    void* base = nullptr;
    int rc = ds.reserve(cv.off + 256, &base);
    if (rc) return rc;
    Carve c;
    c.base = static_cast<char*>(base);
    L = lay(c);
    D.kidOff = c.take<u32>(nnode + 1);
    D.kid = c.take<u32>(nedge);
    D.kidEdge = c.take<u32>(nedge);
    D.up = c.take<u32>(nnode);
    D.down = c.take<u32>(nnode);
    CASPHY_CUDA_TRY(cudaMemcpyAsync(D.kidOff, H.kidOff.data(), 4ull * (nnode + 1), cudaMemcpyHostToDevice, st));
    CASPHY_CUDA_TRY(cudaMemcpyAsync(D.kid, H.kid.data(), 4ull * nedge, cudaMemcpyHostToDevice, st));
    CASPHY_CUDA_TRY(cudaMemcpyAsync(D.kidEdge, H.kidEdge.data(), 4ull * nedge, cudaMemcpyHostToDevice, st));
    CASPHY_CUDA_TRY(cudaMemcpyAsync(D.up, H.upOrder.data(), 4ull * H.upOrder.size(), cudaMemcpyHostToDevice, st));
    CASPHY_CUDA_TRY(cudaMemcpyAsync(D.down, H.downOrder.data(), 4ull * H.downOrder.size(), cudaMemcpyHostToDevice, st));
    return CASPHY_OK;
}

inline u32 blocks(u64 n, u32 t) { return (u32)((n + t - 1) / t); }

}  // namespace

}  // namespace casphy

extern "C" int casphy_ancestral_bit(uint32_t ntip, uint32_t nnode, uint32_t nbin, const uint32_t* mat,
                                    uint32_t nedge, const uint32_t* edge, uint32_t* state_out, uint32_t* edge_len) {
    using namespace casphy;
    int rc = require_device();
    if (rc) return rc;
    if (!mat || !edge_len || nbin == 0 || ntip == 0) return CASPHY_EINVAL;
    HostTree H;
    if ((rc = build(ntip, nnode, nedge, edge, H))) return rc;
    if (H.root != ntip) {
        casphy_set_last_error_msg("parsimony: the root must be node ntip (ape numbering)");
        return CASPHY_EINVAL;
    }
    DeviceScope ds;
    cudaStream_t st = 0;
    struct B {
        u32 *mat, *state, *bis, *conf, *len;
    };
    auto lay = [&](Carve& c) {
        B b;
        b.mat = c.take<u32>((size_t)ntip * nbin);
        b.state = c.take<u32>((size_t)nnode * nbin);
        b.bis = c.take<u32>((size_t)nnode * nbin);
        b.conf = c.take<u32>((size_t)nnode * nbin);
        b.len = c.take<u32>(nedge);
        return b;
    };
    B L;
    DevTree D;
    if ((rc = reserve_and_upload(ds, H, lay, L, D, st))) return rc;
    CASPHY_CUDA_TRY(cudaMemcpyAsync(L.mat, mat, 4ull * ntip * nbin, cudaMemcpyHostToDevice, st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(L.len, 0, 4ull * nedge, st));
    Tree Tu{ntip, D.kidOff, D.kid, D.kidEdge, D.up};
    for (size_t lv = 0; lv + 1 < H.upOff.size(); lv++) {
        const u32 cnt = H.upOff[lv + 1] - H.upOff[lv];
        k_up_bit<<<blocks((u64)cnt * nbin, 256), 256, 0, st>>>(Tu, H.upOff[lv], cnt, nbin, L.mat, L.state, L.bis,
                                                               L.conf);
    }
    k_root_bit<<<blocks(nbin, 256), 256, 0, st>>>(nbin, L.state, L.bis, L.conf);
    Tree Td{ntip, D.kidOff, D.kid, D.kidEdge, D.down};
    for (size_t lv = 0; lv + 1 < H.downOff.size(); lv++) {
        const u32 cnt = H.downOff[lv + 1] - H.downOff[lv];
        k_down_bit<<<blocks((u64)cnt * nbin, 256), 256, 0, st>>>(Td, H.downOff[lv], cnt, nbin, L.mat, L.state, L.bis,
                                                                 L.len);
    }
    CASPHY_CUDA_TRY(cudaGetLastError());
    CASPHY_CUDA_TRY(cudaMemcpyAsync(edge_len, L.len, 4ull * nedge, cudaMemcpyDeviceToHost, st));
    if (state_out)
        CASPHY_CUDA_TRY(cudaMemcpyAsync(state_out, L.state, 4ull * nnode * nbin, cudaMemcpyDeviceToHost, st));
    CASPHY_CUDA_TRY(cudaStreamSynchronize(st));
    return CASPHY_OK;
}

extern "C" int casphy_ancestral_char(uint32_t ntip, uint32_t nnode, uint32_t nsite, const int32_t* mat,
                                     uint32_t nedge, const uint32_t* edge, const uint32_t* tipSize, float minSize,
                                     float minRatio, int32_t* state_out, uint32_t* edge_len) {
    using namespace casphy;
    int rc = require_device();
    if (rc) return rc;
    if (!mat || !edge_len || !tipSize || nsite == 0 || ntip == 0) return CASPHY_EINVAL;
    HostTree H;
    if ((rc = build(ntip, nnode, nedge, edge, H))) return rc;
    // node sizes and the largest child size, then the size rule per edge
    // (charAncestralEC's first loops, src/functions.cpp:3086-3104)
    std::vector<int> nsz(nnode, 0), mx(nnode, 0);
    for (u32 e = nedge; e-- > 0;) {
        const u32 a = edge[2 * e] - ntip, d = edge[2 * e + 1];
        const int sd = d < ntip ? (int)tipSize[d] : nsz[d - ntip];
        nsz[a] += sd;
        if (mx[a] < sd) mx[a] = sd;
    }
    std::vector<unsigned char> use(nedge);
    for (u32 e = 0; e < nedge; e++) {
        const u32 a = edge[2 * e] - ntip, d = edge[2 * e + 1];
        const int sd = d < ntip ? (int)tipSize[d] : nsz[d - ntip];
        use[e] = (minRatio * (float)sd >= (float)mx[a] || (float)sd >= minSize) ? 1 : 0;
    }
    DeviceScope ds;
    cudaStream_t st = 0;
    struct B {
        int *mat, *state;
        u32 *len, *edge;
        unsigned char* use;
    };
    auto lay = [&](Carve& c) {
        B b;
        b.mat = c.take<int>((size_t)ntip * nsite);
        b.state = c.take<int>((size_t)nnode * nsite);
        b.len = c.take<u32>(nedge);
        b.edge = c.take<u32>(2ull * nedge);
        b.use = c.take<unsigned char>(nedge);
        return b;
    };
    B L;
    DevTree D;
    if ((rc = reserve_and_upload(ds, H, lay, L, D, st))) return rc;
    CASPHY_CUDA_TRY(cudaMemcpyAsync(L.mat, mat, 4ull * ntip * nsite, cudaMemcpyHostToDevice, st));
    CASPHY_CUDA_TRY(cudaMemcpyAsync(L.edge, edge, 8ull * nedge, cudaMemcpyHostToDevice, st));
    CASPHY_CUDA_TRY(cudaMemcpyAsync(L.use, use.data(), nedge, cudaMemcpyHostToDevice, st));
    Tree Tu{ntip, D.kidOff, D.kid, D.kidEdge, D.up};
    for (size_t lv = 0; lv + 1 < H.upOff.size(); lv++) {
        const u32 cnt = H.upOff[lv + 1] - H.upOff[lv];
        k_up_char<<<blocks((u64)cnt * nsite, 256), 256, 0, st>>>(Tu, H.upOff[lv], cnt, nsite, L.mat, L.use, L.state);
    }
    k_len_char<<<nedge, 128, 0, st>>>(ntip, nedge, nsite, L.edge, L.mat, L.state, L.len);
    CASPHY_CUDA_TRY(cudaGetLastError());
    CASPHY_CUDA_TRY(cudaMemcpyAsync(edge_len, L.len, 4ull * nedge, cudaMemcpyDeviceToHost, st));
    if (state_out)
        CASPHY_CUDA_TRY(cudaMemcpyAsync(state_out, L.state, 4ull * nnode * nsite, cudaMemcpyDeviceToHost, st));
    CASPHY_CUDA_TRY(cudaStreamSynchronize(st));
    return CASPHY_OK;
}

extern "C" int casphy_node_des(uint32_t ntip, uint32_t nnode, uint32_t nedge, const uint32_t* edge,
                               uint32_t* rows_out, int32_t* sizes_out) {
    using namespace casphy;
    int rc = require_device();
    if (rc) return rc;
    if (!rows_out || !sizes_out || ntip == 0) return CASPHY_EINVAL;
    HostTree H;
    if ((rc = build(ntip, nnode, nedge, edge, H))) return rc;
    const u32 nbin = ((ntip - 1) >> 5) + 1, kCache = 8192;
    // output row of every internal child (reverse edge order), sizes, and the
    // reference's open-row limit (nodeDesBig keeps 8192 cache rows)
    std::vector<u32> rowOf(nnode, nnode - 1);
    std::vector<int> size(nnode, 0);
    std::vector<unsigned char> open(nnode, 0);
    u32 nUse = 0, r = 0;
    for (u32 e = nedge; e-- > 0;) {
        const u32 a = edge[2 * e] - ntip, d = edge[2 * e + 1];
        if (!open[a]) {
            if (nUse == kCache) {
                casphy_set_last_error_msg("Run out of cache!");
                return CASPHY_ERANGE;
            }
            open[a] = 1;
            nUse++;
        }
        if (d < ntip) {
            size[a]++;
        } else {
            size[a] += size[d - ntip];
            rowOf[d - ntip] = r++;
            open[d - ntip] = 0;
            nUse--;
        }
    }
    for (u32 i = 1; i < nnode; i++) sizes_out[nnode - 1 - i] = size[i];
    DeviceScope ds;
    cudaStream_t st = 0;
    struct B {
        u32 *rows, *rowOf;
    };
    auto lay = [&](Carve& c) {
        B b;
        b.rows = c.take<u32>((size_t)nnode * nbin);
        b.rowOf = c.take<u32>(nnode);
        return b;
    };
    B L;
    DevTree D;
    if ((rc = reserve_and_upload(ds, H, lay, L, D, st))) return rc;
    CASPHY_CUDA_TRY(cudaMemcpyAsync(L.rowOf, rowOf.data(), 4ull * nnode, cudaMemcpyHostToDevice, st));
    Tree Tu{ntip, D.kidOff, D.kid, D.kidEdge, D.up};
    for (size_t lv = 0; lv + 1 < H.upOff.size(); lv++) {
        const u32 cnt = H.upOff[lv + 1] - H.upOff[lv];
        k_clade<<<blocks((u64)cnt * nbin, 256), 256, 0, st>>>(Tu, H.upOff[lv], cnt, nbin, L.rowOf, L.rows);
    }
    CASPHY_CUDA_TRY(cudaGetLastError());
    if (nnode > 1)
        CASPHY_CUDA_TRY(cudaMemcpyAsync(rows_out, L.rows, 4ull * (nnode - 1) * nbin, cudaMemcpyDeviceToHost, st));
    CASPHY_CUDA_TRY(cudaStreamSynchronize(st));
    return CASPHY_OK;
}
