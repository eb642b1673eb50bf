// fasta2bin on B200 (replaces cu/fasta2bin.cu, whose work is all on the
// host): the alignment's columns are classified and the kept columns encoded
// on the device.
//
// A column is variable when some base count c (A, T/U, C, G; an IUPAC
// ambiguity code counts for each of its bases, a gap or other character for
// none) has 0 < c < nseq.  The reference tests 0 < c < n after every
// sequence and stops at the first hit (cu/fasta2bin.cu:47-96); counts only
// grow by one per sequence, so that happens exactly when it holds at the end.
// Kept columns are encoded 8 bits per base, four to a u32, low byte first
// (encode_char / encode_sequence, :11-31, :186-206).
#include <vector>

#include "common.cuh"
#include "runtime.h"

namespace casphy {
namespace fasta {

__device__ __forceinline__ u32 base_mask(unsigned char c) {
    switch (c | 0x20) {  // lower case
        case 'a': return 0x1;
        case 't': case 'u': return 0x2;
        case 'c': return 0x4;
        case 'g': return 0x8;
        case 'w': return 0x3;
        case 'm': return 0x5;
        case 'r': return 0x9;
        case 'y': return 0x6;
        case 'k': return 0xA;
        case 's': return 0xC;
        case 'h': return 0x7;
        case 'd': return 0xB;
        case 'v': return 0xD;
        case 'b': return 0xE;
        case 'n': return 0xF;
        default: return 0x10;
    }
}

// one thread per column, sequences in turn (consecutive threads read
// consecutive bytes of one sequence)
__global__ void k_columns(const unsigned char* __restrict__ seq, u32 nseq, u32 len, unsigned char* __restrict__ var) {
    const u32 pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= len) return;
    u32 c0 = 0, c1 = 0, c2 = 0, c3 = 0;
    for (u32 i = 0; i < nseq; i++) {
        const u32 m = base_mask(seq[(size_t)i * len + pos]);
        if (m & 0x10) continue;
        c0 += m & 1u;
        c1 += (m >> 1) & 1u;
        c2 += (m >> 2) & 1u;
        c3 += (m >> 3) & 1u;
    }
    var[pos] = (c0 && c0 < nseq) || (c1 && c1 < nseq) || (c2 && c2 < nseq) || (c3 && c3 < nseq);
}

// one thread per output word: kept columns keep[4w .. 4w+3] of one sequence
__global__ void k_encode(const unsigned char* __restrict__ seq, u32 nseq, u32 len, const u32* __restrict__ keep,
                         u32 nkeep, u32* __restrict__ out) {
    const u32 nw = (nkeep + 3) / 4;
    const u64 id = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= (u64)nseq * nw) return;
    const u32 i = (u32)(id / nw), w = (u32)(id % nw);
    u32 v = 0;
#pragma unroll
    for (u32 j = 0; j < 4; j++) {
        const u32 k = 4 * w + j;
        if (k < nkeep) v |= base_mask(seq[(size_t)i * len + keep[k]]) << (8 * j);
    }
    out[id] = v;
}

}  // namespace fasta
}  // namespace casphy

extern "C" int casphy_fasta_encode(uint32_t nseq, uint32_t len, const char* seqs, uint8_t* variable,
                                   uint32_t* nkeep_out, uint32_t* bin_out, uint64_t bin_cap) {
    using namespace casphy;
    using namespace casphy::fasta;
    int rc = require_device();
    if (rc) return rc;
    if (nseq == 0 || len == 0 || !seqs || !variable || !nkeep_out) return CASPHY_EINVAL;
    DeviceScope ds;
    cudaStream_t st = 0;
    const size_t nch = (size_t)nseq * len;
    const size_t maxWords = (size_t)nseq * ((len + 3) / 4);
    Carve cv;
    cv.take<unsigned char>(nch);
    cv.take<unsigned char>(len);
    cv.take<u32>(len);
    cv.take<u32>(maxWords);
    void* base = nullptr;
    if ((rc = ds.reserve(cv.off + 256, &base))) return rc;
    Carve c;
    c.base = static_cast<char*>(base);
    unsigned char* dseq = c.take<unsigned char>(nch);
    unsigned char* dvar = c.take<unsigned char>(len);
    u32* dkeep = c.take<u32>(len);
    u32* dout = c.take<u32>(maxWords);
    CASPHY_CUDA_TRY(cudaMemcpyAsync(dseq, seqs, nch, cudaMemcpyHostToDevice, st));
    k_columns<<<(len + 255) / 256, 256, 0, st>>>(dseq, nseq, len, dvar);
    CASPHY_CUDA_TRY(cudaGetLastError());
    CASPHY_CUDA_TRY(cudaMemcpyAsync(variable, dvar, len, cudaMemcpyDeviceToHost, st));
    CASPHY_CUDA_TRY(cudaStreamSynchronize(st));
    std::vector<u32> keep;
    for (u32 p = 0; p < len; p++)
        if (variable[p]) keep.push_back(p);
    const u32 nkeep = (u32)keep.size();
    *nkeep_out = nkeep;
    const u64 words = (u64)nseq * ((nkeep + 3) / 4);
    if (!bin_out || nkeep == 0) return CASPHY_OK;
    if (bin_cap < words) return CASPHY_ERANGE;
    CASPHY_CUDA_TRY(cudaMemcpyAsync(dkeep, keep.data(), 4ull * nkeep, cudaMemcpyHostToDevice, st));
    k_encode<<<(unsigned)((words + 255) / 256), 256, 0, st>>>(dseq, nseq, len, dkeep, nkeep, dout);
    CASPHY_CUDA_TRY(cudaGetLastError());
    CASPHY_CUDA_TRY(cudaMemcpyAsync(bin_out, dout, 4ull * words, cudaMemcpyDeviceToHost, st));
    CASPHY_CUDA_TRY(cudaStreamSynchronize(st));
    return CASPHY_OK;
}
