// TransferDisStream on B200 (replaces cu/TransferDisStream.cu).
//
// For clade bitsets X (nrow_x rows) and Y (nrow_y rows) over ntip tips packed
// in ncol u32 words, the reference keeps, per x row, the minimum over y of
// min(d, c - pad) with d = popc(x ^ y), c = popc(x ^ ~y) = 32*ncol - d and
// pad = 32*ncol - ntip, but forms the two minima separately over aligned
// groups of 8 y rows before subtracting pad (u32 arithmetic), and seeds
// missing rows of a partial group with 32*ncol (cu/TransferDisStream.cu:
// 39-104); y rows symmetrically over groups of 8 x rows.  That grouping
// changes the result only when rows carry bits past ntip, and it is kept
// exactly.  Sizes are min(k, ntip - k), k = popcount of the row (:107-121).
//
// One launch tiles 32 x rows (lanes) by 64 y rows (8 warps x one group of
// 8), streams 32-word chunks of both tiles through shared memory, and keeps
// the 8 distances per thread in registers; x minima are reduced across the
// warps, y minima across aligned 8-lane segments, then merged with atomicMin.
#include <vector>

#include "common.cuh"
#include "runtime.h"

namespace casphy {
namespace tdis {

constexpr u32 kTX = 32, kTY = 64, kChunk = 32;

__global__ void __launch_bounds__(256) k_cross(const u32* __restrict__ X, const u32* __restrict__ Y, u32 nx, u32 ny,
                                               u32 ncol, u32 ntip, u32* __restrict__ xmin, u32* __restrict__ ymin) {
    __shared__ u32 xs[kTX][kChunk + 1];
    __shared__ u32 ys[kTY][kChunk];
    __shared__ u32 red[8][kTX];
    const u32 lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const u32 x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY;
    u32 d[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (u32 k0 = 0; k0 < ncol; k0 += kChunk) {
        const u32 kn = min(kChunk, ncol - k0);
        for (u32 i = threadIdx.x; i < kTX * kChunk; i += 256) {
            const u32 r = i / kChunk, k = i % kChunk;
            xs[r][k] = (x0 + r < nx && k < kn) ? X[(size_t)(x0 + r) * ncol + k0 + k] : 0u;
        }
        for (u32 i = threadIdx.x; i < kTY * kChunk; i += 256) {
            const u32 r = i / kChunk, k = i % kChunk;
            ys[r][k] = (y0 + r < ny && k < kn) ? Y[(size_t)(y0 + r) * ncol + k0 + k] : 0u;
        }
        __syncthreads();
        for (u32 k = 0; k < kn; k++) {
            const u32 xv = xs[lane][k];
#pragma unroll
            for (int i = 0; i < 8; i++) d[i] += (u32)__popc(xv ^ ys[w * 8 + i][k]);
        }
        __syncthreads();
    }
    const u32 full = 32u * ncol, pad = 32u * ncol - ntip;
    const bool xok = x0 + lane < nx;
    // x side: this thread's 8 y rows are one aligned group
    {
        u32 A = full, B = full;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            if (y0 + w * 8 + i < ny) {
                A = min(A, d[i]);
                B = min(B, full - d[i]);
            }
        }
        const u32 t2 = B - pad;
        red[w][lane] = A > t2 ? t2 : A;
        __syncthreads();
        if (w == 0 && xok) {
            u32 v = red[0][lane];
            for (int g = 1; g < 8; g++)
                if (y0 + g * 8 < ny) v = min(v, red[g][lane]);
            atomicMin(xmin + x0 + lane, v);
        }
    }
    // y side: aligned groups of 8 lanes are groups of 8 x rows
#pragma unroll
    for (int i = 0; i < 8; i++) {
        u32 A = xok ? d[i] : full;
        u32 B = xok ? full - d[i] : full;
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            A = min(A, __shfl_xor_sync(0xFFFFFFFFu, A, o));
            B = min(B, __shfl_xor_sync(0xFFFFFFFFu, B, o));
        }
        const u32 y = y0 + w * 8 + i;
        if ((lane & 7) == 0 && y < ny && x0 + lane < nx) {
            const u32 t2 = B - pad;
            atomicMin(ymin + y, A > t2 ? t2 : A);
        }
    }
}

__global__ void k_sizes(const u32* __restrict__ M, u32 n, u32 ncol, u32 ntip, u32* __restrict__ size) {
    const u32 r = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const u32 lane = threadIdx.x & 31;
    if (r >= n) return;
    u32 c = 0;
    for (u32 k = lane; k < ncol; k += 32) c += (u32)__popc(M[(size_t)r * ncol + k]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
    if (lane == 0) size[r] = c > ntip - c ? ntip - c : c;
}

__global__ void k_fill_u32(u32* p, u32 n, u32 v) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

}  // namespace tdis

int transfer_dis_device(u32 ny, u32 nx, u32 ncol, u32 ntip, const u32* dY, const u32* dX, u32* dYmin, u32* dYsize,
                        u32* dXmin, u32* dXsize, cudaStream_t st) {
    using namespace tdis;
    const u32 full = 32u * ncol;
    if (ny) k_fill_u32<<<(ny + 255) / 256, 256, 0, st>>>(dYmin, ny, full);
    if (nx) k_fill_u32<<<(nx + 255) / 256, 256, 0, st>>>(dXmin, nx, full);
    if (nx && ny) k_cross<<<dim3((nx + kTX - 1) / kTX, (ny + kTY - 1) / kTY), 256, 0, st>>>(dX, dY, nx, ny, ncol, ntip,
                                                                                           dXmin, dYmin);
    if (ny) k_sizes<<<(ny + 7) / 8, 256, 0, st>>>(dY, ny, ncol, ntip, dYsize);
    if (nx) k_sizes<<<(nx + 7) / 8, 256, 0, st>>>(dX, nx, ncol, ntip, dXsize);
    CASPHY_CUDA_TRY(cudaGetLastError());
    return CASPHY_OK;
}

}  // namespace casphy

extern "C" int casphy_transfer_dis(uint32_t nrow_y, uint32_t nrow_x, uint32_t ncol, uint32_t ntip, const uint32_t* y,
                                   const uint32_t* x, uint32_t* ymin, uint32_t* ysize, uint32_t* xmin,
                                   uint32_t* xsize) {
    using namespace casphy;
    int rc = require_device();
    if (rc) return rc;
    if (ncol == 0 || (nrow_y && (!y || !ymin || !ysize)) || (nrow_x && (!x || !xmin || !xsize))) return CASPHY_EINVAL;
    DeviceScope ds;
    cudaStream_t st = 0;
    auto lay = [&](Carve& c) {
        struct B { u32* y; u32* x; u32* ymin; u32* ysize; u32* xmin; u32* xsize; } b;
        b.y = c.take<u32>((size_t)nrow_y * ncol);
        b.x = c.take<u32>((size_t)nrow_x * ncol);
        b.ymin = c.take<u32>(nrow_y);
        b.ysize = c.take<u32>(nrow_y);
        b.xmin = c.take<u32>(nrow_x);
        b.xsize = c.take<u32>(nrow_x);
        return b;
    };
    Carve cv;
    lay(cv);
    void* base = nullptr;
    rc = ds.reserve(cv.off + 256, &base);
    if (rc) return rc;
    Carve c2;
    c2.base = static_cast<char*>(base);
    auto L = lay(c2);
    if (nrow_y) CASPHY_CUDA_TRY(cudaMemcpyAsync(L.y, y, sizeof(u32) * (size_t)nrow_y * ncol, cudaMemcpyHostToDevice, st));
    if (nrow_x) CASPHY_CUDA_TRY(cudaMemcpyAsync(L.x, x, sizeof(u32) * (size_t)nrow_x * ncol, cudaMemcpyHostToDevice, st));
    rc = transfer_dis_device(nrow_y, nrow_x, ncol, ntip, L.y, L.x, L.ymin, L.ysize, L.xmin, L.xsize, st);
    if (rc) return rc;
    if (nrow_y) {
        CASPHY_CUDA_TRY(cudaMemcpyAsync(ymin, L.ymin, sizeof(u32) * nrow_y, cudaMemcpyDeviceToHost, st));
        CASPHY_CUDA_TRY(cudaMemcpyAsync(ysize, L.ysize, sizeof(u32) * nrow_y, cudaMemcpyDeviceToHost, st));
    }
    if (nrow_x) {
        CASPHY_CUDA_TRY(cudaMemcpyAsync(xmin, L.xmin, sizeof(u32) * nrow_x, cudaMemcpyDeviceToHost, st));
        CASPHY_CUDA_TRY(cudaMemcpyAsync(xsize, L.xsize, sizeof(u32) * nrow_x, cudaMemcpyDeviceToHost, st));
    }
    CASPHY_CUDA_TRY(cudaStreamSynchronize(st));
    return CASPHY_OK;
}
