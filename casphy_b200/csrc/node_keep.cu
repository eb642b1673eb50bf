// nodeKeepIndel / nodeKeepBit on B200 (replaces cu/nodeKeepIndel.cu and
// cu/nodeKeepBit.cu).
//
// The reference walks the pre-order edge list and, for each internal child
// not inside an already kept node, launches one kernel over the out-group
// rows and copies the counts back (cu/nodeKeepIndel.cu:132-152).  Whether a
// node passes the test does not depend on the walk, only whether it is
// tested does.  So one launch tests every internal node against every
// out-group row (one CTA per node, out-group rows column-major so the
// threads of a CTA read consecutive rows; a CTA stops at the first row under
// the cutoff), and the host replays the walk with the skip rule.
#include <vector>

#include "common.cuh"
#include "runtime.h"

namespace casphy {
namespace nodekeep {

constexpr int kThreads = 256;

// outT[s * nRetain + j] = outmat[j * ncol + s]
__global__ void k_transpose_u32(const u32* __restrict__ in, u32 rows, u32 cols, u32* __restrict__ out) {
    __shared__ u32 tile[32][33];
    const u32 r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    for (u32 r = threadIdx.y; r < 32; r += blockDim.y)
        if (r0 + r < rows && c0 + threadIdx.x < cols) tile[r][threadIdx.x] = in[(size_t)(r0 + r) * cols + c0 + threadIdx.x];
    __syncthreads();
    for (u32 c = threadIdx.y; c < 32; c += blockDim.y)
        if (c0 + c < cols && r0 + threadIdx.x < rows) out[(size_t)(c0 + c) * rows + r0 + threadIdx.x] = tile[threadIdx.x][c];
}

// keep[v] = 1 when every out-group row j has count(v, j) >= cutoff.
// BIT: count = popc(node & ~row) (cu/nodeKeepBit.cu:33-51); otherwise
// count = #{i : node_i > 1, row_i != node_i, row_i >= 1} (cu/nodeKeepIndel.cu:32-48).
template <bool BIT>
__global__ void __launch_bounds__(kThreads) k_keep(const u32* __restrict__ nodeState, u32 nnode, u32 ncol,
                                                   const u32* __restrict__ outT, u32 nRetain, u32 cutoff,
                                                   unsigned char* __restrict__ keep) {
    extern __shared__ u32 sm[];
    u32* eIdx = sm;          // ncol
    u32* eVal = sm + ncol;   // ncol
    __shared__ u32 s_n, s_fail;
    const u32 v = blockIdx.x;
    if (v >= nnode) return;
    if (threadIdx.x == 0) { s_n = 0; s_fail = 0; }
    __syncthreads();
    const u32* ref = nodeState + (size_t)v * ncol;
    for (u32 i = threadIdx.x; i < ncol; i += kThreads) {
        const u32 r = ref[i];
        const bool use = BIT ? r != 0u : r > 1u;
        if (use) {
            const u32 pos = atomicAdd(&s_n, 1u);
            eIdx[pos] = i;
            eVal[pos] = r;
        }
    }
    __syncthreads();
    const u32 n = s_n;
    for (u32 j0 = 0; j0 < nRetain; j0 += kThreads) {
        const u32 j = j0 + threadIdx.x;
        if (j < nRetain) {
            u32 cnt = 0;
            for (u32 e = 0; e < n; e++) {
                const u32 x = outT[(size_t)eIdx[e] * nRetain + j];
                const u32 r = eVal[e];
                if (BIT) cnt += (u32)__popc(r & ~x);
                else cnt += (x != r && x >= 1u) ? 1u : 0u;
            }
            if (cnt < cutoff) s_fail = 1;
        }
        __syncthreads();
        if (s_fail) break;
    }
    if (threadIdx.x == 0) keep[v] = s_fail ? 0 : 1;
}

}  // namespace nodekeep

// Replays the reference walk (cu/nodeKeepIndel.cu:130-152) over the edge
// list with the per-node verdicts.
static int node_keep_impl(bool bit, u32 nnodeRows, u32 ncol, const u32* nodeState, u32 nedge, const u32* edge,
                          u32 nRetain, const u32* outmat, u32 cutoff, u32* out_nodes, u32* nout) {
    using namespace nodekeep;
    if (!nodeState || !edge || !out_nodes || !nout || ncol == 0) return CASPHY_EINVAL;
    if (nRetain && !outmat) return CASPHY_EINVAL;
    const u32 ntip = nnodeRows + 1;
    std::vector<unsigned char> keep(nnodeRows ? nnodeRows : 1, 1);
    if (nRetain > 0 && nnodeRows > 0) {
        if (sizeof(u32) * 2 * (size_t)ncol > 200 * 1024) {
            casphy_set_last_error_msg("nodeKeep: too many columns for the per-node site list");
            return CASPHY_ERANGE;
        }
        DeviceScope ds;
        Carve cv;
        auto lay = [&](Carve& c) {
            struct B { u32* ns; u32* om; u32* omT; unsigned char* keep; } b;
            b.ns = c.take<u32>((size_t)nnodeRows * ncol);
            b.om = c.take<u32>((size_t)nRetain * ncol);
            b.omT = c.take<u32>((size_t)nRetain * ncol);
            b.keep = c.take<unsigned char>(nnodeRows);
            return b;
        };
        lay(cv);
        void* base = nullptr;
        int rc = ds.reserve(cv.off + 256, &base);
        if (rc) return rc;
        Carve c2;
        c2.base = static_cast<char*>(base);
        auto L = lay(c2);
        cudaStream_t st = 0;
        CASPHY_CUDA_TRY(cudaMemcpyAsync(L.ns, nodeState, sizeof(u32) * (size_t)nnodeRows * ncol, cudaMemcpyHostToDevice, st));
        CASPHY_CUDA_TRY(cudaMemcpyAsync(L.om, outmat, sizeof(u32) * (size_t)nRetain * ncol, cudaMemcpyHostToDevice, st));
        k_transpose_u32<<<dim3((nRetain + 31) / 32, (ncol + 31) / 32), dim3(32, 8), 0, st>>>(L.om, nRetain, ncol, L.omT);
        const size_t smem = sizeof(u32) * 2 * ncol;
        if (bit) {
            CASPHY_CUDA_TRY(cudaFuncSetAttribute(k_keep<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k_keep<true><<<nnodeRows, kThreads, smem, st>>>(L.ns, nnodeRows, ncol, L.omT, nRetain, cutoff, L.keep);
        } else {
            CASPHY_CUDA_TRY(cudaFuncSetAttribute(k_keep<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k_keep<false><<<nnodeRows, kThreads, smem, st>>>(L.ns, nnodeRows, ncol, L.omT, nRetain, cutoff, L.keep);
        }
        CASPHY_CUDA_TRY(cudaGetLastError());
        CASPHY_CUDA_TRY(cudaMemcpyAsync(keep.data(), L.keep, nnodeRows, cudaMemcpyDeviceToHost, st));
        CASPHY_CUDA_TRY(cudaStreamSynchronize(st));
    }
    u32 currentNode = ntip - 1, flag = 0, n = 0;
    for (u32 i = 0; i < nedge; i++) {
        const u32 parent = edge[2 * i], child = edge[2 * i + 1];
        if (!(child + 1 > ntip)) continue;
        if (flag == 1 && currentNode <= parent) continue;
        const u32 row = child - ntip;
        if (row >= nnodeRows) {
            casphy_set_last_error_msg("nodeKeep: edge references a node beyond the state rows");
            return CASPHY_ERANGE;
        }
        flag = keep[row];
        if (flag) {
            currentNode = child;
            out_nodes[n++] = child;
        }
    }
    *nout = n;
    return CASPHY_OK;
}

}  // namespace casphy

extern "C" int casphy_node_keep_indel(uint32_t nnodeRows, uint32_t ncol, const uint32_t* nodeState, uint32_t nedge,
                                      const uint32_t* edge, uint32_t nRetain, const uint32_t* outmat, uint32_t cutoff,
                                      uint32_t* out_nodes, uint32_t* nout) {
    int rc = casphy::require_device();
    if (rc) return rc;
    return casphy::node_keep_impl(false, nnodeRows, ncol, nodeState, nedge, edge, nRetain, outmat, cutoff, out_nodes,
                                  nout);
}

extern "C" int casphy_node_keep_bit(uint32_t nnodeRows, uint32_t nbin, const uint32_t* nodeState, uint32_t nedge,
                                    const uint32_t* edge, uint32_t nRetain, const uint32_t* outmat, uint32_t cutoff,
                                    uint32_t* out_nodes, uint32_t* nout) {
    int rc = casphy::require_device();
    if (rc) return rc;
    return casphy::node_keep_impl(true, nnodeRows, nbin, nodeState, nedge, edge, nRetain, outmat, cutoff, out_nodes,
                                  nout);
}
