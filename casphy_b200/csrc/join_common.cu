// Kernels and host helpers shared by the indel and bit joins.
#include <vector>

#include "join_engine.cuh"

namespace casphy {
namespace joinx {

__global__ void k_slot_init(u32 ntip, u32 Sp, u32 nnode, const unsigned long long* initKey, u32 ordNeg1, u32* lmOrd,
                            u32* lmIdx, u32* slotNode, u32* node2slot, u32* nodeDeath, u32* nodeSize,
                            const u32* tipSize) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < Sp) {
        if (i < ntip) {
            const u64 k = initKey[i];
            lmOrd[i] = key_ord(k);
            lmIdx[i] = key_node(k);
            slotNode[i] = i;
        } else {
            lmOrd[i] = ordNeg1;
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

// Pre-order walk of the raw join edges (cu/joinEdgeIndel.cu:488-558): node v's
// edges are 2(v-ntip) (first child) and 2(v-ntip)+1; the root is 2ntip-2.
// Writes the relabelled edge list and, in `order`, the node of every state
// row (root first, then internal nodes in discovery order).
void preorder_relabel(u32 ntip, const u32* rawEdge, u32* edge_out, u32* order) {
    const u32 nnode = 2 * ntip - 1;
    std::vector<u32> relabel(nnode), stack;
    std::vector<unsigned char> cursor(nnode, 0);
    for (u32 i = 0; i < nnode; i++) relabel[i] = i < ntip ? i : nnode;
    stack.reserve(nnode);
    u32 nord = 0, count = ntip, nout = 0;
    order[nord++] = nnode - 1;
    stack.push_back(nnode - 1);
    while (!stack.empty()) {
        const u32 v = stack.back();
        if (v < ntip || cursor[v] >= 2) { stack.pop_back(); continue; }
        const u32 ei = 2 * (v - ntip) + cursor[v];
        cursor[v]++;
        const u32 p = rawEdge[2 * ei], c = rawEdge[2 * ei + 1];
        stack.push_back(c);
        if (relabel[p] == nnode) relabel[p] = count++;
        if (relabel[c] == nnode) {
            order[nord++] = c;
            relabel[c] = count++;
        }
        edge_out[2 * nout] = relabel[p];
        edge_out[2 * nout + 1] = relabel[c];
        nout++;
    }
}

}  // namespace joinx
}  // namespace casphy
