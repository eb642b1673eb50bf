// Bootstrap column resampling of fasta2bin matrices (replaces the gather of
// cu/Felsenstein.cu:34-54): output byte j of word i of a row is the input
// byte at position idx[4i+j] (positions count bytes, 4 per u32 word).
#include "common.cuh"
#include "runtime.h"

namespace casphy {
namespace resample {

__global__ void k_gather_bytes(const u32* __restrict__ in, u32 ntip, u32 nbin, const u32* __restrict__ idx, u32 nidx,
                               u32* __restrict__ out) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;  // output word
    const u32 nout = (nidx + 3) / 4;
    if (i >= nout) return;
    u32 t[4];
#pragma unroll
    for (u32 j = 0; j < 4; j++) t[j] = 4 * i + j < nidx ? idx[4 * i + j] : 0xFFFFFFFFu;
    for (u32 row = blockIdx.y; row < ntip; row += gridDim.y) {
        const u32* src = in + (size_t)row * nbin;
        u32 v = 0;
#pragma unroll
        for (u32 j = 0; j < 4; j++)
            if ((t[j] >> 2) < nbin) v |= ((__ldg(src + (t[j] >> 2)) >> ((t[j] & 3) * 8)) & 0xFFu) << (j * 8);
        out[(size_t)row * nout + i] = v;
    }
}

}  // namespace resample
}  // namespace casphy

extern "C" int casphy_resample_columns(uint32_t ntip, uint32_t nbin, const uint32_t* in, uint32_t nidx,
                                       const uint32_t* idx, uint32_t* out) {
    using namespace casphy;
    int rc = require_device();
    if (rc) return rc;
    if ((ntip && (!in || !out)) || (nidx && !idx)) return CASPHY_EINVAL;
    const u32 nout = (nidx + 3) / 4;
    if (ntip == 0 || nout == 0) return CASPHY_OK;
    DeviceScope ds;
    Carve cv;
    cv.take<u32>((size_t)ntip * nbin);
    cv.take<u32>(nidx);
    cv.take<u32>((size_t)ntip * nout);
    void* base = nullptr;
    rc = ds.reserve(cv.off + 256, &base);
    if (rc) return rc;
    Carve c;
    c.base = static_cast<char*>(base);
    u32* dIn = c.take<u32>((size_t)ntip * nbin);
    u32* dIdx = c.take<u32>(nidx);
    u32* dOut = c.take<u32>((size_t)ntip * nout);
    cudaStream_t st = 0;
    CASPHY_CUDA_TRY(cudaMemcpyAsync(dIn, in, sizeof(u32) * (size_t)ntip * nbin, cudaMemcpyHostToDevice, st));
    CASPHY_CUDA_TRY(cudaMemcpyAsync(dIdx, idx, sizeof(u32) * nidx, cudaMemcpyHostToDevice, st));
    resample::k_gather_bytes<<<dim3((nout + 127) / 128, ntip < 65535 ? ntip : 65535), 128, 0, st>>>(dIn, ntip, nbin, dIdx, nidx, dOut);
    CASPHY_CUDA_TRY(cudaGetLastError());
    CASPHY_CUDA_TRY(cudaMemcpyAsync(out, dOut, sizeof(u32) * (size_t)ntip * nout, cudaMemcpyDeviceToHost, st));
    CASPHY_CUDA_TRY(cudaStreamSynchronize(st));
    return CASPHY_OK;
}
