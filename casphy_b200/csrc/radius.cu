// Radius neighbour search on B200: radiusNeighbor, radiusNeighborDNA,
// tryRadius and tryRadiusDNA (replaces the cu/ files of those names).
//
// The reference tests one query row at a time against the rows after its
// 32-row block and mirrors the hits on the host (cu/radiusNeighbor.cu:
// 331-425); its output is, for every row i, the ascending list of rows j with
// score(i, j) >= radius (the score is symmetric), and the list sizes.
//   bit rows:  score = sum of w[b] over the bits set in both rows, binary32,
//              ascending bit order (:33-41); unit weights -> popcount.
//   DNA rows:  score = number of positions whose 4-bit IUPAC codes intersect
//              (cu/radiusNeighborDNA.cu:55-87).  Here the codes are stored as
//              four bit planes per block of 32 positions (plane j = bit j of
//              the code), so one block costs popc((q0&c0)|(q1&c1)|(q2&c2)|
//              (q3&c3)): nine integer operations for 32 positions.
// Here the whole neighbour relation is produced as a bit matrix in one
// tiled all-pairs launch (32 query rows per CTA in shared memory x 256
// candidate rows, one warp ballot per 32 candidates), rows are counted, and
// a second launch expands the bits into the ascending index lists.
#include <sys/mman.h>

#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "runtime.h"

namespace casphy {
namespace radius {

// Host buffer for lists the library allocates (released with free()).  A large
// one is 2 MiB-aligned and advised into transparent huge pages: the pageable
// device-to-host copy then faults it in 2 MiB at a time instead of 4 KiB (for
// 10,000 rows that all neighbour each other, 400 MB: ~200 faults, not ~100,000).
static u32* alloc_lists(u64 n) {
    constexpr size_t kHuge = size_t(2) << 20;
    const size_t bytes = sizeof(u32) * (n ? n : 1);
    if (bytes < 2 * kHuge) return static_cast<u32*>(std::malloc(bytes));
    const size_t rounded = (bytes + kHuge - 1) / kHuge * kHuge;
    void* p = std::aligned_alloc(kHuge, rounded);
    if (p) madvise(p, rounded, MADV_HUGEPAGE);  // advice only: a refusal leaves 4 KiB pages
    return static_cast<u32*>(p);
}

constexpr int kThreads = 256;  // candidates per CTA
constexpr int kQ = 32;         // query rows per CTA
enum { SC_UNIT = 0, SC_FLOAT = 1, SC_DNA = 2 };

// rows are column-major: word k of row t at col[k * ld + t]
template <int MODE>
__global__ void __launch_bounds__(kThreads) k_mask(const u32* __restrict__ col, u32 nwords, u32 ld, u32 ntip,
                                                   u32 qBegin, u32 qEnd, const float* __restrict__ wf, float radius,
                                                   u32 uradius, u32 maskWords, u32* __restrict__ mask) {
    extern __shared__ __align__(16) u32 qs[];  // kQ x nwords query words (query rows qBegin..qEnd-1)
    const u32 q0 = qBegin + blockIdx.y * kQ;
    const u32 t = blockIdx.x * kThreads + threadIdx.x;
    for (u32 i = threadIdx.x; i < kQ * nwords; i += kThreads) {
        const u32 q = i / nwords, k = i % nwords;
        qs[q * nwords + k] = q0 + q < qEnd ? col[(size_t)k * ld + q0 + q] : 0u;
    }
    __syncthreads();
    u32 acc[kQ];
    float facc[kQ];
#pragma unroll
    for (int q = 0; q < kQ; q++) {
        acc[q] = 0u;
        facc[q] = 0.0f;
    }
    if (t < ntip && MODE == SC_DNA) {
        // blocks of 32 positions, four plane words each
        const uint4* q4 = reinterpret_cast<const uint4*>(qs);
        const u32 nblk = nwords / 4;
        for (u32 b = 0; b < nblk; b++) {
            const u32 c0 = col[(size_t)(4 * b) * ld + t], c1 = col[(size_t)(4 * b + 1) * ld + t];
            const u32 c2 = col[(size_t)(4 * b + 2) * ld + t], c3 = col[(size_t)(4 * b + 3) * ld + t];
#pragma unroll
            for (int q = 0; q < kQ; q++) {
                const uint4 v = q4[q * nblk + b];
                acc[q] += (u32)__popc((v.x & c0) | (v.y & c1) | (v.z & c2) | (v.w & c3));
            }
        }
    } else if (t < ntip) {
        for (u32 k = 0; k < nwords; k++) {
            const u32 c = col[(size_t)k * ld + t];
            if (MODE == SC_UNIT) {
#pragma unroll
                for (int q = 0; q < kQ; q++) acc[q] += (u32)__popc(qs[q * nwords + k] & c);
            } else {
#pragma unroll
                for (int q = 0; q < kQ; q++) {
                    u32 m = qs[q * nwords + k] & c;
                    while (m) {
                        const int b = __ffs(m) - 1;
                        facc[q] += __ldg(wf + k * 32 + b);
                        m &= m - 1;
                    }
                }
            }
        }
    }
    const u32 lane = threadIdx.x & 31;
#pragma unroll
    for (int q = 0; q < kQ; q++) {
        bool hit;
        if (MODE == SC_UNIT) hit = (float)acc[q] >= radius;
        else if (MODE == SC_DNA) hit = acc[q] >= uradius;
        else hit = facc[q] >= radius;
        hit = hit && t < ntip;
        const u32 bal = __ballot_sync(0xFFFFFFFFu, hit);
        if (lane == 0 && q0 + q < qEnd && (t >> 5) < maskWords)
            mask[(size_t)(q0 + q - qBegin) * maskWords + (t >> 5)] = bal;
    }
}

// counts[i] = popcount of row i of the mask
__global__ void k_count(const u32* __restrict__ mask, u32 ntip, u32 maskWords, u32* __restrict__ counts) {
    const u32 row = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const u32 lane = threadIdx.x & 31;
    if (row >= ntip) return;
    u32 n = 0;
    for (u32 w = lane; w < maskWords; w += 32) n += (u32)__popc(mask[(size_t)row * maskWords + w]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xFFFFFFFFu, n, o);
    if (lane == 0) counts[row] = n;
}

// idx[off[i] ...] = ascending set bits of row i (one warp per row)
__global__ void k_expand(const u32* __restrict__ mask, u32 ntip, u32 maskWords, const u64* __restrict__ off,
                         u32* __restrict__ idx) {
    const u32 row = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const u32 lane = threadIdx.x & 31;
    if (row >= ntip) return;
    u64 o = off[row];
    for (u32 w0 = 0; w0 < maskWords; w0 += 32) {
        const u32 w = w0 + lane;
        u32 m = w < maskWords ? mask[(size_t)row * maskWords + w] : 0u;
        const u32 c = __popc(m);
        u32 incl = c;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const u32 v = __shfl_up_sync(0xFFFFFFFFu, incl, d);
            if (lane >= (u32)d) incl += v;
        }
        u64 p = o + incl - c;
        while (m) {
            const int b = __ffs(m) - 1;
            idx[p++] = w * 32 + b;
            m &= m - 1;
        }
        o += __shfl_sync(0xFFFFFFFFu, incl, 31);
    }
}

// fasta2bin bytes -> column-major bit planes: for block b of 32 positions,
// word 4b+j holds bit j of the low nibble of the code of position 32b+s at
// bit s (the reference keeps the same low nibbles, packed eight to a word,
// cu/radiusNeighborDNA.cu:27-53).
__global__ void k_pack_dna(const u32* __restrict__ raw, u32 ntip, u32 nbinRaw, u32 nblk, u32 ld,
                           u32* __restrict__ col) {
    const u32 t = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 b = blockIdx.y;
    if (t >= ntip || b >= nblk) return;
    u32 p[4] = {0u, 0u, 0u, 0u};
    for (u32 h = 0; h < 8; h++) {
        const u32 wi = 8 * b + h;
        if (wi >= nbinRaw) break;
        const u32 r = raw[(size_t)t * nbinRaw + wi];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const u32 code = (r >> (8 * i)) & 0xFu, s = 4 * h + i;
#pragma unroll
            for (int j = 0; j < 4; j++) p[j] |= ((code >> j) & 1u) << s;
        }
    }
#pragma unroll
    for (int j = 0; j < 4; j++) col[(size_t)(4 * b + j) * ld + t] = p[j];
}

// tryRadius: counts[r] = #{t < ntip : score(q_r, t) >= radius}; bit rows
// with radius <= 0 also count the idle threads of the last 128-thread block
// (cu/tryRadius.cu:44-49).
template <int MODE>
__global__ void k_try(const u32* __restrict__ col, u32 nwords, u32 ld, u32 ntip, const float* __restrict__ wf,
                      float radius, u32 uradius, const u32* __restrict__ qidx, u32* __restrict__ counts) {
    const u32 r = blockIdx.y;
    const u32 t = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 q = qidx[r];
    bool hit = false;
    if (t < ntip && MODE == SC_DNA) {
        u32 acc = 0;
        for (u32 b = 0; b < nwords / 4; b++) {
            u32 x = 0;
#pragma unroll
            for (int j = 0; j < 4; j++) x |= col[(size_t)(4 * b + j) * ld + q] & col[(size_t)(4 * b + j) * ld + t];
            acc += (u32)__popc(x);
        }
        hit = acc >= uradius;
    } else if (t < ntip) {
        u32 acc = 0;
        float facc = 0.f;
        for (u32 k = 0; k < nwords; k++) {
            const u32 x = col[(size_t)k * ld + q] & col[(size_t)k * ld + t];
            if (MODE == SC_UNIT) acc += (u32)__popc(x);
            else {
                u32 m = x;
                while (m) {
                    const int b = __ffs(m) - 1;
                    facc += __ldg(wf + k * 32 + b);
                    m &= m - 1;
                }
            }
        }
        if (MODE == SC_UNIT) hit = (float)acc >= radius;
        else hit = facc >= radius;
    }
    const u32 bal = __ballot_sync(0xFFFFFFFFu, hit);
    if ((threadIdx.x & 31) == 0 && bal) atomicAdd(counts + r, (u32)__popc(bal));
}

}  // namespace radius

using namespace radius;

struct RadiusInput {
    bool dna;
    u32 ntip, nwords;  // words per row (bit rows: nrow; DNA: 4 plane words per 32 positions)
    const u32* hostWordPlane;  // bit rows, word-plane-major (the .bmat body)
    const u32* hostRaw;        // DNA rows, fasta2bin layout
    u32 nbinRaw;
    std::vector<float> wf;
    int mode;
    float radius;
    u32 uradius;
};

// Uploads rows column-major (ld = ntip); returns the device pointer.
static int upload_rows(const RadiusInput& in, Carve& c, u32** col, float** wf, cudaStream_t st) {
    *col = c.take<u32>((size_t)in.nwords * in.ntip);
    *wf = c.take<float>(in.wf.size() ? in.wf.size() : 1);
    if (in.dna) {
        u32* raw = c.take<u32>((size_t)in.ntip * in.nbinRaw);
        CASPHY_CUDA_TRY(cudaMemcpyAsync(raw, in.hostRaw, sizeof(u32) * (size_t)in.ntip * in.nbinRaw,
                                        cudaMemcpyHostToDevice, st));
        k_pack_dna<<<dim3((in.ntip + 255) / 256, in.nwords / 4), 256, 0, st>>>(raw, in.ntip, in.nbinRaw, in.nwords / 4,
                                                                               in.ntip, *col);
    } else {
        CASPHY_CUDA_TRY(cudaMemcpyAsync(*col, in.hostWordPlane, sizeof(u32) * (size_t)in.nwords * in.ntip,
                                        cudaMemcpyHostToDevice, st));
    }
    if (in.wf.size())
        CASPHY_CUDA_TRY(cudaMemcpyAsync(*wf, in.wf.data(), sizeof(float) * in.wf.size(), cudaMemcpyHostToDevice, st));
    return CASPHY_OK;
}

static int prep_bit(RadiusInput& in, u32 nrow, u32 ntip, const u32* bmat, const double* w, int32_t radius) {
    if (!bmat || !w || ntip == 0 || nrow == 0) return CASPHY_EINVAL;
    in.dna = false;
    in.ntip = ntip;
    in.nwords = nrow;
    in.hostWordPlane = bmat;
    in.wf.resize((size_t)nrow * 32);
    bool unit = true;
    for (size_t i = 0; i < in.wf.size(); i++) {
        in.wf[i] = (float)w[i];
        if (in.wf[i] != 1.0f) unit = false;
    }
    in.mode = unit ? SC_UNIT : SC_FLOAT;
    if (unit) in.wf.clear();
    in.radius = (float)radius;
    in.uradius = 0;
    return CASPHY_OK;
}

static int prep_dna(RadiusInput& in, u32 ntip, u32 nbinRaw, const u32* raw, u32 radius) {
    if (!raw || ntip == 0 || nbinRaw == 0) return CASPHY_EINVAL;
    in.dna = true;
    in.ntip = ntip;
    in.nbinRaw = nbinRaw;
    in.hostRaw = raw;
    in.nwords = 4 * ((nbinRaw + 7) / 8);  // 32 positions = 8 raw words per block
    in.mode = SC_DNA;
    in.radius = 0;
    in.uradius = radius;
    return CASPHY_OK;
}

// Lists of the query rows [row0, row1) (counts[0 .. row1-row0) and their
// concatenated index lists); the whole matrix is [0, ntip).
// allocOut non-null: the lists go to a host buffer of the exact size,
// allocated here once they are counted (freed with casphy_free).
static int radius_impl(RadiusInput& in, u32 row0, u32 row1, u32* counts, u32* idx, u64 cap, u64* total,
                       u32** allocOut = nullptr) {
    if (!counts || row0 > row1 || row1 > in.ntip) return CASPHY_EINVAL;
    const u32 ntip = in.ntip, nq = row1 - row0;
    if (allocOut) *allocOut = nullptr;
    if (nq == 0) {
        if (total) *total = 0;
        if (allocOut) *allocOut = static_cast<u32*>(std::malloc(sizeof(u32)));
        return allocOut && !*allocOut ? CASPHY_ENOMEM : CASPHY_OK;
    }
    const u32 maskWords = (ntip + 31) / 32;
    const size_t smem = sizeof(u32) * kQ * in.nwords;
    if (smem > 200 * 1024) {
        casphy_set_last_error_msg("radius: rows too wide for the shared-memory query tile");
        return CASPHY_ERANGE;
    }
    DeviceScope ds;
    cudaStream_t st = 0;
    auto lay = [&](Carve& c) {
        struct B { u32* mask; u32* counts; u64* off; } b;
        b.mask = c.take<u32>((size_t)nq * maskWords);
        b.counts = c.take<u32>(nq);
        b.off = c.take<u64>(nq);
        return b;
    };
    // sizes: rows + mask first; index space after counting
    Carve cv;
    u32* dcol;
    float* dwf;
    cv.take<u32>((size_t)in.nwords * ntip);
    cv.take<float>(in.wf.size() ? in.wf.size() : 1);
    if (in.dna) cv.take<u32>((size_t)ntip * in.nbinRaw);
    lay(cv);
    const size_t base0 = cv.off;
    void* base = nullptr;
    int rc = ds.reserve(base0 + 256, &base);
    if (rc) return rc;
    Carve c2;
    c2.base = static_cast<char*>(base);
    rc = upload_rows(in, c2, &dcol, &dwf, st);
    if (rc) return rc;
    auto L = lay(c2);
    dim3 grid((ntip + kThreads - 1) / kThreads, (nq + kQ - 1) / kQ);
    void* fn = in.mode == SC_UNIT ? (void*)k_mask<SC_UNIT> : in.mode == SC_DNA ? (void*)k_mask<SC_DNA>
                                                                                  : (void*)k_mask<SC_FLOAT>;
    CASPHY_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (in.mode == SC_UNIT)
        k_mask<SC_UNIT><<<grid, kThreads, smem, st>>>(dcol, in.nwords, ntip, ntip, row0, row1, dwf, in.radius, in.uradius,
                                                       maskWords, L.mask);
    else if (in.mode == SC_DNA)
        k_mask<SC_DNA><<<grid, kThreads, smem, st>>>(dcol, in.nwords, ntip, ntip, row0, row1, dwf, in.radius, in.uradius,
                                                      maskWords, L.mask);
    else
        k_mask<SC_FLOAT><<<grid, kThreads, smem, st>>>(dcol, in.nwords, ntip, ntip, row0, row1, dwf, in.radius, in.uradius,
                                                        maskWords, L.mask);
    k_count<<<(nq + 7) / 8, 256, 0, st>>>(L.mask, nq, maskWords, L.counts);
    CASPHY_CUDA_TRY(cudaGetLastError());
    CASPHY_CUDA_TRY(cudaMemcpyAsync(counts, L.counts, sizeof(u32) * nq, cudaMemcpyDeviceToHost, st));
    CASPHY_CUDA_TRY(cudaStreamSynchronize(st));
    std::vector<u64> off(nq);
    u64 tot = 0;
    for (u32 i = 0; i < nq; i++) {
        off[i] = tot;
        tot += counts[i];
    }
    if (total) *total = tot;
    if (allocOut) {
        idx = alloc_lists(tot);
        if (!idx) return CASPHY_ENOMEM;
        cap = tot;
        *allocOut = idx;
    }
    if (!idx) return CASPHY_OK;
    if (tot > cap) return CASPHY_ERANGE;
    // the index lists get the second block: their size is only known now
    void* auxp = nullptr;
    if ((rc = ds.reserve_aux(sizeof(u32) * (tot ? tot : 1), &auxp))) return rc;
    u32* didx = static_cast<u32*>(auxp);
    CASPHY_CUDA_TRY(cudaMemcpyAsync(L.off, off.data(), sizeof(u64) * nq, cudaMemcpyHostToDevice, st));
    k_expand<<<(nq + 7) / 8, 256, 0, st>>>(L.mask, nq, maskWords, L.off, didx);
    CASPHY_CUDA_TRY(cudaGetLastError());
    if (tot) CASPHY_CUDA_TRY(cudaMemcpyAsync(idx, didx, sizeof(u32) * tot, cudaMemcpyDeviceToHost, st));
    CASPHY_CUDA_TRY(cudaStreamSynchronize(st));
    return CASPHY_OK;
}

static int try_impl(RadiusInput& in, u32 nrep, const u32* qidx, u32* counts) {
    if (!counts || (nrep && !qidx)) return CASPHY_EINVAL;
    for (u32 r = 0; r < nrep; r++)
        if (qidx[r] >= in.ntip) return CASPHY_ERANGE;
    if (nrep == 0) return CASPHY_OK;
    DeviceScope ds;
    cudaStream_t st = 0;
    Carve cv;
    cv.take<u32>((size_t)in.nwords * in.ntip);
    cv.take<float>(in.wf.size() ? in.wf.size() : 1);
    if (in.dna) cv.take<u32>((size_t)in.ntip * in.nbinRaw);
    cv.take<u32>(nrep);
    cv.take<u32>(nrep);
    void* base = nullptr;
    int rc = ds.reserve(cv.off + 256, &base);
    if (rc) return rc;
    Carve c2;
    c2.base = static_cast<char*>(base);
    u32* dcol;
    float* dwf;
    rc = upload_rows(in, c2, &dcol, &dwf, st);
    if (rc) return rc;
    u32* dq = c2.take<u32>(nrep);
    u32* dc = c2.take<u32>(nrep);
    CASPHY_CUDA_TRY(cudaMemcpyAsync(dq, qidx, sizeof(u32) * nrep, cudaMemcpyHostToDevice, st));
    CASPHY_CUDA_TRY(cudaMemsetAsync(dc, 0, sizeof(u32) * nrep, st));
    dim3 grid((in.ntip + 255) / 256, nrep);
    if (in.mode == SC_UNIT)
        k_try<SC_UNIT><<<grid, 256, 0, st>>>(dcol, in.nwords, in.ntip, in.ntip, dwf, in.radius, in.uradius, dq, dc);
    else if (in.mode == SC_DNA)
        k_try<SC_DNA><<<grid, 256, 0, st>>>(dcol, in.nwords, in.ntip, in.ntip, dwf, in.radius, in.uradius, dq, dc);
    else
        k_try<SC_FLOAT><<<grid, 256, 0, st>>>(dcol, in.nwords, in.ntip, in.ntip, dwf, in.radius, in.uradius, dq, dc);
    CASPHY_CUDA_TRY(cudaGetLastError());
    CASPHY_CUDA_TRY(cudaMemcpyAsync(counts, dc, sizeof(u32) * nrep, cudaMemcpyDeviceToHost, st));
    CASPHY_CUDA_TRY(cudaStreamSynchronize(st));
    if (!in.dna && in.radius <= 0.0f) {
        const u32 pad = (in.ntip + 127u) / 128u * 128u - in.ntip;
        for (u32 r = 0; r < nrep; r++) counts[r] += pad;
    }
    return CASPHY_OK;
}

}  // namespace casphy

extern "C" int casphy_radius_bit(uint32_t nrow, uint32_t ntip, const uint32_t* bmat, const double* weight,
                                 int32_t radius, uint32_t* counts, uint32_t* idx, uint64_t idx_cap, uint64_t* total) {
    int rc = casphy::require_device();
    if (rc) return rc;
    casphy::RadiusInput in;
    rc = casphy::prep_bit(in, nrow, ntip, bmat, weight, radius);
    if (rc) return rc;
    return casphy::radius_impl(in, 0, ntip, counts, idx, idx_cap, total);
}

extern "C" int casphy_radius_bit_rows(uint32_t nrow, uint32_t ntip, const uint32_t* bmat, const double* weight,
                                      int32_t radius, uint32_t row_begin, uint32_t row_end, uint32_t* counts,
                                      uint32_t* idx, uint64_t idx_cap, uint64_t* total) {
    int rc = casphy::require_device();
    if (rc) return rc;
    casphy::RadiusInput in;
    rc = casphy::prep_bit(in, nrow, ntip, bmat, weight, radius);
    if (rc) return rc;
    return casphy::radius_impl(in, row_begin, row_end, counts, idx, idx_cap, total);
}

extern "C" int casphy_radius_dna(uint32_t ntip, uint32_t nbinRaw, const uint32_t* raw, uint32_t radius,
                                 uint32_t* counts, uint32_t* idx, uint64_t idx_cap, uint64_t* total) {
    int rc = casphy::require_device();
    if (rc) return rc;
    casphy::RadiusInput in;
    rc = casphy::prep_dna(in, ntip, nbinRaw, raw, radius);
    if (rc) return rc;
    return casphy::radius_impl(in, 0, ntip, counts, idx, idx_cap, total);
}

extern "C" int casphy_radius_dna_rows(uint32_t ntip, uint32_t nbinRaw, const uint32_t* raw, uint32_t radius,
                                      uint32_t row_begin, uint32_t row_end, uint32_t* counts, uint32_t* idx,
                                      uint64_t idx_cap, uint64_t* total) {
    int rc = casphy::require_device();
    if (rc) return rc;
    casphy::RadiusInput in;
    rc = casphy::prep_dna(in, ntip, nbinRaw, raw, radius);
    if (rc) return rc;
    return casphy::radius_impl(in, row_begin, row_end, counts, idx, idx_cap, total);
}

extern "C" int casphy_radius_bit_lists(uint32_t nrow, uint32_t ntip, const uint32_t* bmat, const double* weight,
                                       int32_t radius, uint32_t* counts, uint32_t** idx_out, uint64_t* total) {
    int rc = casphy::require_device();
    if (rc) return rc;
    if (!idx_out) return CASPHY_EINVAL;
    casphy::RadiusInput in;
    rc = casphy::prep_bit(in, nrow, ntip, bmat, weight, radius);
    if (rc) return rc;
    rc = casphy::radius_impl(in, 0, ntip, counts, nullptr, 0, total, idx_out);
    if (rc && *idx_out) {
        std::free(*idx_out);
        *idx_out = nullptr;
    }
    return rc;
}

extern "C" int casphy_radius_dna_lists(uint32_t ntip, uint32_t nbinRaw, const uint32_t* raw, uint32_t radius,
                                       uint32_t* counts, uint32_t** idx_out, uint64_t* total) {
    int rc = casphy::require_device();
    if (rc) return rc;
    if (!idx_out) return CASPHY_EINVAL;
    casphy::RadiusInput in;
    rc = casphy::prep_dna(in, ntip, nbinRaw, raw, radius);
    if (rc) return rc;
    rc = casphy::radius_impl(in, 0, ntip, counts, nullptr, 0, total, idx_out);
    if (rc && *idx_out) {
        std::free(*idx_out);
        *idx_out = nullptr;
    }
    return rc;
}

extern "C" void casphy_free(void* p) { std::free(p); }

extern "C" int casphy_try_radius_bit(uint32_t nrow, uint32_t ntip, const uint32_t* bmat, const double* weight,
                                     int32_t radius, uint32_t nrep, const uint32_t* qidx, uint32_t* counts) {
    int rc = casphy::require_device();
    if (rc) return rc;
    casphy::RadiusInput in;
    rc = casphy::prep_bit(in, nrow, ntip, bmat, weight, radius);
    if (rc) return rc;
    return casphy::try_impl(in, nrep, qidx, counts);
}

extern "C" int casphy_try_radius_dna(uint32_t ntip, uint32_t nbinRaw, const uint32_t* raw, uint32_t radius,
                                     uint32_t nrep, const uint32_t* qidx, uint32_t* counts) {
    int rc = casphy::require_device();
    if (rc) return rc;
    casphy::RadiusInput in;
    rc = casphy::prep_dna(in, ntip, nbinRaw, raw, radius);
    if (rc) return rc;
    return casphy::try_impl(in, nrep, qidx, counts);
}
