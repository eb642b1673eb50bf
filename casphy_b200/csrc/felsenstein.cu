// Felsenstein pruning with an adjoint gradient, and branch-length
// optimisation, on B200.
//
// CasPhy has no likelihood code (its cu/Felsenstein.cu is the bootstrap
// column resampler, see resample.cu; branch lengths there are parsimony
// change counts, src/functions.cpp:3480-3542).  This component follows
// Felsenstein (1981).  Partial likelihoods are binary32 with an exact
// power-of-two renormalisation per (node, site), the exponent carried as an
// integer; the per-site log likelihood and its sum are binary64.
//
// Inside pass: internal nodes grouped by height, one launch per height, one
// thread per (node, site).  Outside pass: internal nodes grouped by depth,
// one launch per depth; for each child edge c of node p it forms
// R = U_p * M_sibling and the site term w_s (R . dM_c/dt) / (R . M_c) of
// d log L / d t_c, then passes U_c = R P_c down.  Both ratios are invariant
// to the scale of R, so outside vectors are renormalised freely.  Site terms
// are reduced per block and written to a per-(edge, site block) array that a
// last kernel sums in a fixed order (site terms in binary32 within a block,
// the blocks in binary64), so log L and the gradient are bitwise
// reproducible.  Sites are processed in chunks whose partials fit a
// device-memory budget (sites are independent, so nothing is recomputed).
// All launches of one evaluation are captured once per problem into a CUDA
// graph and replayed for every evaluation.
//
// Branch lengths are optimised over x = log t by L-BFGS in binary64 on the
// device: the two-loop recursion and the history update run as cooperative
// one-CTA-per-SM kernels whose grid reductions sum per-CTA partials in a
// fixed order behind a bounded flag barrier; the host only reads back the
// scalars the Armijo line search needs.  The "plain" variant replaces the
// adjoint gradient by per-edge central differences of log L (2 evaluations
// per edge) and is otherwise identical.
//
// Models: HKY85 (Hasegawa, Kishino & Yano 1985) on the 4-bit IUPAC nibble of
// fasta2bin (bit 0 A, 1 T, 2 C, 3 G; an empty nibble is missing data) and an
// irreversible edit model for CRISPR indels (state 0 unedited, alleles a >= 1;
// P(0->0) = exp(-r t), P(0->a) = q_a (1 - exp(-r t)), alleles never change;
// the root is unedited).  For the edit model a (node, site) partial is
// (L0, La, allele): La is non-zero for at most the one allele consistent with
// the subtree, or for every allele alike when the subtree is missing at the
// site, so two floats and an allele id represent it exactly; the outside
// vector is (U0, X, Y, allele) with U(a) = X q_a + Y [a == allele].
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "runtime.h"

namespace casphy {
namespace fel {

constexpr u32 kSites = 256;  // sites per block (one thread per site)
constexpr int kWild = 0x7FFF, kNoneA = 0x7FFE;
constexpr u32 kLbThreads = 512;
constexpr u32 kMaxLbCTA = 256;  // CTAs of the cooperative L-BFGS kernels
constexpr u32 kMaxHist = 16;

struct Tree {
    u32 ntip;
    const u32* kidA;  // per internal node (index v - ntip)
    const u32* kidB;
    const u32* edgeA;
    const u32* edgeB;
    const u32* inOrder;   // internal nodes by height
    const u32* outOrder;  // internal nodes by depth
    const uint4* inInfo;  // per position of inOrder: {node, kidA, kidB, edgeA}
    const u32* inEdgeB;   // per position of inOrder: edgeB
    const uint4* outInfo; // per position of outOrder
    const u32* outEdgeB;
};

// 2^-e with e the exponent of m (m > 0, normal, not near the top of the
// range): returned in sc, exactly; false sends the caller to ilogbf/ldexpf.
__device__ __forceinline__ bool pow2_of(float m, int& e, float& sc) {
    const int ex = (__float_as_int(m) >> 23) & 0xFF;
    if (ex < 1 || ex > 253) return false;
    e = ex - 127;
    sc = __int_as_float((254 - ex) << 23);
    return true;
}

// One chunk of sites [s0, s0 + w); partial buffers have row stride W.
struct Chunk {
    u32 s0, w, W, nsite, blk0, nblkTot;
};

__device__ __forceinline__ double block_sum(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0;
    if (threadIdx.x == 0)
        for (u32 i = 0; i < blockDim.x / 32; i++) t += red[i];
    return t;  // valid in thread 0
}

// Block sums of two binary32 values (thread 0 gets them); one CTA barrier
// pair for both children's site terms.
__device__ __forceinline__ float2 block_sum2f(float a, float b, float2* red) {
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xFFFFFFFFu, a, o);
        b += __shfl_xor_sync(0xFFFFFFFFu, b, o);
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = make_float2(a, b);
    __syncthreads();
    float2 t = make_float2(0.f, 0.f);
    if (threadIdx.x == 0)
        for (u32 i = 0; i < blockDim.x / 32; i++) {
            t.x += red[i].x;
            t.y += red[i].y;
        }
    return t;
}

// ---------------------------------------------------------------- HKY85 ---

struct Hky {
    double lam[4];
    double V[16];
    double Vi[16];
    double pi[4];
};

__global__ void k_pmat_hky(const double* __restrict__ t, u32 nedge, Hky m, float* __restrict__ P,
                           float* __restrict__ dP) {
    pdl_wait();
    pdl_trigger();
    const u32 e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nedge) return;
    double ex[4], dx[4];
    for (int k = 0; k < 4; k++) {
        ex[k] = exp(m.lam[k] * t[e]);
        dx[k] = m.lam[k] * ex[k];
    }
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            double a = 0, b = 0;
            for (int k = 0; k < 4; k++) {
                a += m.V[i * 4 + k] * ex[k] * m.Vi[k * 4 + j];
                b += m.V[i * 4 + k] * dx[k] * m.Vi[k * 4 + j];
            }
            // store P - I: O(t) entries with full relative precision, so the
            // binary32 rounding is not one shared error across all sites
            P[e * 16 + i * 4 + j] = (float)(i == j ? a - 1.0 : fmax(a, 0.0));
            dP[e * 16 + i * 4 + j] = (float)b;
        }
}

__device__ __forceinline__ float4 tip_hky(u32 code) {
    const u32 n = code & 0xFu;
    if (n == 0) return make_float4(1.f, 1.f, 1.f, 1.f);
    return make_float4((float)(n & 1u), (float)((n >> 1) & 1u), (float)((n >> 2) & 1u), (float)((n >> 3) & 1u));
}

__device__ __forceinline__ float4 matvec(const float* __restrict__ P, float4 x) {
    return make_float4(P[0] * x.x + P[1] * x.y + P[2] * x.z + P[3] * x.w,
                       P[4] * x.x + P[5] * x.y + P[6] * x.z + P[7] * x.w,
                       P[8] * x.x + P[9] * x.y + P[10] * x.z + P[11] * x.w,
                       P[12] * x.x + P[13] * x.y + P[14] * x.z + P[15] * x.w);
}

// (I + D) x and r^T (I + D) for D = P - I
__device__ __forceinline__ float4 pmatvec(const float* __restrict__ D, float4 x) {
    const float4 d = matvec(D, x);
    return make_float4(x.x + d.x, x.y + d.y, x.z + d.z, x.w + d.w);
}

__device__ __forceinline__ float4 pvecmat(float4 r, const float* __restrict__ D) {
    return make_float4(r.x + (r.x * D[0] + r.y * D[4] + r.z * D[8] + r.w * D[12]),
                       r.y + (r.x * D[1] + r.y * D[5] + r.z * D[9] + r.w * D[13]),
                       r.z + (r.x * D[2] + r.y * D[6] + r.z * D[10] + r.w * D[14]),
                       r.w + (r.x * D[3] + r.y * D[7] + r.z * D[11] + r.w * D[15]));
}

__device__ __forceinline__ float dot4(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }

// exact power-of-two renormalisation of the largest entry to [1, 2)
__device__ __forceinline__ int renorm4(float4& v) {
    const float m = fmaxf(fmaxf(v.x, v.y), fmaxf(v.z, v.w));
    if (!(m > 0.f)) return 0;
    int e;
    float sc;
    if (pow2_of(m, e, sc)) {
        v.x *= sc;
        v.y *= sc;
        v.z *= sc;
        v.w *= sc;
        return e;
    }
    e = ilogbf(m);
    v.x = ldexpf(v.x, -e);
    v.y = ldexpf(v.y, -e);
    v.z = ldexpf(v.z, -e);
    v.w = ldexpf(v.w, -e);
    return e;
}

struct HkyBuf {
    const u32* codes;  // ntip x nsite
    float4* L;         // nint x W
    int* E;            // nint x W
    float4* U;         // nint x W
    const float* P;   // per edge P - I (row-major 4x4)
    const float* dP;  // per edge dP/dt
};

__device__ __forceinline__ float4 child_hky(const Tree& T, const HkyBuf& B, const Chunk& C, u32 c, u32 s, int* e) {
    if (c < T.ntip) {
        *e = 0;
        return tip_hky(__ldg(B.codes + (size_t)c * C.nsite + C.s0 + s));
    }
    const size_t i = (size_t)(c - T.ntip) * C.W + s;
    *e = B.E[i];
    return B.L[i];
}

// One (node, site) of the inside pass once its children's partials are in.
__device__ __forceinline__ void inside_hky_site(const HkyBuf& B, const Chunk& C, u32 vi, u32 eA, u32 eB, u32 s,
                                                float4 la, int ea, float4 lb, int eb) {
    const float4 ma = pmatvec(B.P + 16 * eA, la);
    const float4 mb = pmatvec(B.P + 16 * eB, lb);
    float4 l = make_float4(ma.x * mb.x, ma.y * mb.y, ma.z * mb.z, ma.w * mb.w);
    const int e = renorm4(l);
    B.L[(size_t)vi * C.W + s] = l;
    B.E[(size_t)vi * C.W + s] = ea + eb + e;
}

// 128 threads per 256-site block, two sites per thread (128 apart), every
// child load issued before any arithmetic
__global__ void __launch_bounds__(kSites / 2) k_inside_hky(Tree T, HkyBuf B, Chunk C, u32 off) {
    pdl_wait();
    pdl_trigger();
    const uint4 nf = T.inInfo[off + blockIdx.y];
    const u32 vi = nf.x - T.ntip, eB = T.inEdgeB[off + blockIdx.y];
    u32 sj[2];
    float4 la[2], lb[2];
    int ea[2], eb[2];
#pragma unroll
    for (int j = 0; j < 2; j++) {
        sj[j] = blockIdx.x * kSites + threadIdx.x + j * (kSites / 2);
        const u32 ss = sj[j] < C.w ? sj[j] : 0u;
        la[j] = child_hky(T, B, C, nf.y, ss, &ea[j]);
        lb[j] = child_hky(T, B, C, nf.z, ss, &eb[j]);
    }
#pragma unroll
    for (int j = 0; j < 2; j++)
        if (sj[j] < C.w) inside_hky_site(B, C, vi, nf.w, eB, sj[j], la[j], ea[j], lb[j], eb[j]);
}

__global__ void __launch_bounds__(kSites) k_loglik_hky(u32 root, Tree T, HkyBuf B, Chunk C, Hky m,
                                                       const double* __restrict__ w, double* part) {
    pdl_wait();
    pdl_trigger();
    __shared__ double red[kSites / 32];
    const u32 s = blockIdx.x * kSites + threadIdx.x;
    double v = 0.0;
    if (s < C.w) {
        int e;
        const float4 l = child_hky(T, B, C, root, s, &e);
        const double site = m.pi[0] * (double)l.x + m.pi[1] * (double)l.y + m.pi[2] * (double)l.z +
                            m.pi[3] * (double)l.w;
        v = w[C.s0 + s] * (log(site) + (double)e * 0.69314718055994530942);
    }
    v = block_sum(v, red);
    if (threadIdx.x == 0) part[C.blk0 + blockIdx.x] = v;
}

__global__ void __launch_bounds__(kSites / 2, 10) k_outside_hky(u32 root, Tree T, HkyBuf B, Chunk C, u32 off, Hky m,
                                                        const double* __restrict__ w, double* gpart) {
    pdl_wait();
    pdl_trigger();
    __shared__ float sm[64];
    const uint4 nf = T.outInfo[off + blockIdx.y];
    const u32 v = nf.x, vi = v - T.ntip;
    const u32 ca = nf.y, cb = nf.z;
    const u32 eA = nf.w, eB = T.outEdgeB[off + blockIdx.y];
    if (threadIdx.x < 64) {
        const u32 q = threadIdx.x >> 4, i = threadIdx.x & 15;
        const u32 ed = (q & 1) ? eB : eA;
        sm[threadIdx.x] = __ldg((q < 2 ? B.P : B.dP) + 16 * ed + i);
    }
    // two sites per thread, 128 apart: all loads first
    u32 sj[2], ssj[2];
    bool okj[2];
    float4 u[2], la[2], lb[2];
    int e;
#pragma unroll
    for (int j = 0; j < 2; j++) {
        sj[j] = blockIdx.x * kSites + threadIdx.x + j * (kSites / 2);
        okj[j] = sj[j] < C.w;
        ssj[j] = okj[j] ? sj[j] : 0;
        if (v == root) u[j] = make_float4((float)m.pi[0], (float)m.pi[1], (float)m.pi[2], (float)m.pi[3]);
        else u[j] = B.U[(size_t)vi * C.W + ssj[j]];
        la[j] = child_hky(T, B, C, ca, ssj[j], &e);
        lb[j] = child_hky(T, B, C, cb, ssj[j], &e);
    }
    __syncthreads();
    float gs[2][2] = {{0.f, 0.f}, {0.f, 0.f}};  // [side][j]
#pragma unroll
    for (int j = 0; j < 2; j++) {
        const float4 ma = pmatvec(sm, la[j]), mb = pmatvec(sm + 16, lb[j]);
        const float ws = okj[j] ? (float)w[C.s0 + sj[j]] : 0.f;
#pragma unroll
        for (int side = 0; side < 2; side++) {
            const u32 c = side ? cb : ca;
            const float4 msib = side ? ma : mb;
            const float4 lc = side ? lb[j] : la[j];
            const float4 mc = side ? mb : ma;
            const float4 r = make_float4(u[j].x * msib.x, u[j].y * msib.y, u[j].z * msib.z, u[j].w * msib.w);
            const float4 dm = matvec(sm + 32 + 16 * side, lc);
            gs[side][j] = okj[j] ? ws * (dot4(r, dm) / dot4(r, mc)) : 0.f;
            if (okj[j] && c >= T.ntip) {
                float4 uc = pvecmat(r, sm + 16 * side);
                renorm4(uc);
                B.U[(size_t)(c - T.ntip) * C.W + sj[j]] = uc;
            }
        }
    }
    // site terms in binary32 within the block, grouped as 32-site warps in
    // site order (warp w of half j holds sites 128 j + 32 w ..); blocks are
    // added in binary64
    __shared__ float2 red8[kSites / 32];
#pragma unroll
    for (int j = 0; j < 2; j++) {
        float a = gs[0][j], b = gs[1][j];
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xFFFFFFFFu, a, o);
            b += __shfl_xor_sync(0xFFFFFFFFu, b, o);
        }
        if ((threadIdx.x & 31) == 0) red8[(threadIdx.x >> 5) + j * (kSites / 64)] = make_float2(a, b);
    }
    __syncthreads();
    float2 g = make_float2(0.f, 0.f);
    if (threadIdx.x == 0)
        for (u32 i = 0; i < kSites / 32; i++) {
            g.x += red8[i].x;
            g.y += red8[i].y;
        }
    if (threadIdx.x == 0) {
        gpart[(size_t)eA * C.nblkTot + C.blk0 + blockIdx.x] = g.x;
        gpart[(size_t)eB * C.nblkTot + C.blk0 + blockIdx.x] = g.y;
    }
}

// ------------------------------------------------------- irreversible ---
// partial: float4 {L0, La, allele (int bits), exponent (int bits)}
// outside: float4 {U0, X, Y, allele (int bits)}

struct IrrBuf {
    const u32* codes;  // ntip x nsite (.tbmat coding)
    float4* L;         // nint x W
    float4* U;         // nint x W
    const float2* p;   // per edge (exp(-r t), 1 - exp(-r t))
    const float* q;    // nsite x qstride allele frequencies (index = allele)
    u32 qstride;
    float rate;
};

__device__ __forceinline__ float4 tip_irr(u32 code) {
    if (code == 0) return make_float4(1.f, 1.f, __int_as_float(kWild), 0.f);
    if (code == 1) return make_float4(1.f, 0.f, __int_as_float(kNoneA), 0.f);
    return make_float4(0.f, 1.f, __int_as_float((int)code - 1), 0.f);
}

__device__ __forceinline__ float4 child_irr(const Tree& T, const IrrBuf& B, const Chunk& C, u32 c, u32 s) {
    if (c < T.ntip) return tip_irr(__ldg(B.codes + (size_t)c * C.nsite + C.s0 + s));
    return B.L[(size_t)(c - T.ntip) * C.W + s];
}

__device__ __forceinline__ float qof(const IrrBuf& B, u32 gs, int a) { return __ldg(B.q + (size_t)gs * B.qstride + a); }

// sum_a q_a La(a) of a partial
__device__ __forceinline__ float qsum(const IrrBuf& B, u32 gs, float4 l) {
    const int a = __float_as_int(l.z);
    if (a == kWild) return l.y;
    if (a == kNoneA) return 0.f;
    return qof(B, gs, a) * l.y;
}

__global__ void k_pmat_irr(const double* __restrict__ t, u32 nedge, double rate, float2* __restrict__ p) {
    pdl_wait();
    pdl_trigger();
    const u32 e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < nedge) p[e] = make_float2((float)exp(-rate * t[e]), (float)(-expm1(-rate * t[e])));
}

// One (node, site) of the inside pass once its children's partials are in.
__device__ __forceinline__ void inside_irr_site(const IrrBuf& B, const Chunk& C, u32 vi, float2 pa, float2 pb, u32 s,
                                                float4 la, float4 lb) {
    const u32 gs = C.s0 + s;
    const float m0a = la.x + pa.y * (qsum(B, gs, la) - la.x);
    const float m0b = lb.x + pb.y * (qsum(B, gs, lb) - lb.x);
    const int aa = __float_as_int(la.z), ab = __float_as_int(lb.z);
    float l0 = m0a * m0b, lA = 0.f;
    int a = kNoneA;
    if (aa != kNoneA && ab != kNoneA) {
        if (aa == kWild) a = ab;
        else if (ab == kWild || aa == ab) a = aa;
        if (a != kNoneA) lA = la.y * lb.y;
        if (lA == 0.f) a = kNoneA;
    }
    int e = 0;
    const float mx = fmaxf(l0, lA);
    if (mx > 0.f) {
        float sc;
        if (pow2_of(mx, e, sc)) {
            l0 *= sc;
            lA *= sc;
        } else {
            e = ilogbf(mx);
            l0 = ldexpf(l0, -e);
            lA = ldexpf(lA, -e);
        }
    }
    e += __float_as_int(la.w) + __float_as_int(lb.w);
    B.L[(size_t)vi * C.W + s] = make_float4(l0, lA, __int_as_float(a), __int_as_float(e));
}

// 128 threads per 256-site block, two sites per thread (128 apart), every
// child load issued before any arithmetic
__global__ void __launch_bounds__(kSites / 2) k_inside_irr(Tree T, IrrBuf B, Chunk C, u32 off) {
    pdl_wait();
    pdl_trigger();
    const uint4 nf = T.inInfo[off + blockIdx.y];
    const u32 vi = nf.x - T.ntip;
    const float2 pa = B.p[nf.w], pb = B.p[T.inEdgeB[off + blockIdx.y]];
    u32 sj[2];
    float4 la[2], lb[2];
#pragma unroll
    for (int j = 0; j < 2; j++) {
        sj[j] = blockIdx.x * kSites + threadIdx.x + j * (kSites / 2);
        const u32 ss = sj[j] < C.w ? sj[j] : 0u;
        la[j] = child_irr(T, B, C, nf.y, ss);
        lb[j] = child_irr(T, B, C, nf.z, ss);
    }
#pragma unroll
    for (int j = 0; j < 2; j++)
        if (sj[j] < C.w) inside_irr_site(B, C, vi, pa, pb, sj[j], la[j], lb[j]);
}

__global__ void __launch_bounds__(kSites) k_loglik_irr(u32 root, Tree T, IrrBuf B, Chunk C,
                                                       const double* __restrict__ w, double* part) {
    pdl_wait();
    pdl_trigger();
    __shared__ double red[kSites / 32];
    const u32 s = blockIdx.x * kSites + threadIdx.x;
    double v = 0.0;
    if (s < C.w) {
        const float4 l = child_irr(T, B, C, root, s);
        v = w[C.s0 + s] * (log((double)l.x) + (double)__float_as_int(l.w) * 0.69314718055994530942);
    }
    v = block_sum(v, red);
    if (threadIdx.x == 0) part[C.blk0 + blockIdx.x] = v;
}

__global__ void __launch_bounds__(kSites) k_outside_irr(u32 root, Tree T, IrrBuf B, Chunk C, u32 off,
                                                        const double* __restrict__ w, double* gpart) {
    pdl_wait();
    pdl_trigger();
    __shared__ float2 red[kSites / 32];
    const u32 s = blockIdx.x * kSites + threadIdx.x;
    const uint4 nf = T.outInfo[off + blockIdx.y];
    const u32 v = nf.x, vi = v - T.ntip;
    const bool ok = s < C.w;
    const u32 ss = ok ? s : 0, gs = C.s0 + ss;
    float U0 = 1.f, X = 0.f, Y = 0.f;
    int aY = kNoneA;
    if (v != root) {
        const float4 u = B.U[(size_t)vi * C.W + ss];
        U0 = u.x;
        X = u.y;
        Y = u.z;
        aY = __float_as_int(u.w);
    }
    const u32 kids[2] = {nf.y, nf.z};
    const u32 eds[2] = {nf.w, T.outEdgeB[off + blockIdx.y]};
    float4 l[2];
    float m0[2], qs[2];
    float2 pp[2];
#pragma unroll
    for (int i = 0; i < 2; i++) {
        l[i] = child_irr(T, B, C, kids[i], ss);
        pp[i] = B.p[eds[i]];
        qs[i] = qsum(B, gs, l[i]);
        m0[i] = l[i].x + pp[i].y * (qs[i] - l[i].x);
    }
    const float ws = ok ? (float)w[gs] : 0.f;
    float gsum[2];
#pragma unroll
    for (int c = 0; c < 2; c++) {
        const int sb = 1 - c;
        // R = U * M_sibling
        const float R0 = U0 * m0[sb];
        const int asb = __float_as_int(l[sb].z);
        float RX = 0.f, RY = 0.f;
        int aR = kNoneA;
        if (asb == kWild) {
            RX = l[sb].y * X;
            RY = l[sb].y * Y;
            aR = aY;
        } else if (asb != kNoneA) {
            RY = l[sb].y * (X * qof(B, gs, asb) + (asb == aY ? Y : 0.f));
            aR = asb;
        }
        const int ac = __float_as_int(l[c].z);
        const float dm0 = B.rate * pp[c].x * (qs[c] - l[c].x);
        float den = R0 * m0[c];
        if (ac == kWild) den += l[c].y * (RX + (aR != kNoneA ? RY : 0.f));
        else if (ac != kNoneA) den += l[c].y * (RX * qof(B, gs, ac) + (aR == ac ? RY : 0.f));
        gsum[c] = ok ? ws * ((R0 * dm0) / den) : 0.f;
        if (ok && kids[c] >= T.ntip) {
            float u0 = R0 * pp[c].x, x = pp[c].y * R0 + RX, y = RY;
            const float mx = fmaxf(u0, fmaxf(x, y));
            if (mx > 0.f) {
                int ee;
                float sc;
                if (pow2_of(mx, ee, sc)) {
                    u0 *= sc;
                    x *= sc;
                    y *= sc;
                } else {
                    ee = ilogbf(mx);
                    u0 = ldexpf(u0, -ee);
                    x = ldexpf(x, -ee);
                    y = ldexpf(y, -ee);
                }
            }
            B.U[(size_t)(kids[c] - T.ntip) * C.W + s] = make_float4(u0, x, y, __int_as_float(aR));
        }
    }
    // site terms in binary32 within the block; blocks are added in binary64
    const float2 g = block_sum2f(gsum[0], gsum[1], red);
    if (threadIdx.x == 0) {
        gpart[(size_t)eds[0] * C.nblkTot + C.blk0 + blockIdx.x] = g.x;
        gpart[(size_t)eds[1] * C.nblkTot + C.blk0 + blockIdx.x] = g.y;
    }
}

// ------------------------------------------------ fixed-order reductions ---

__global__ void k_sum_ll(const double* __restrict__ part, u32 n, double* out) {
    pdl_wait();
    pdl_trigger();
    __shared__ double red[32];
    double v = 0;
    // each thread sums a contiguous run, then runs are added in thread order
    const u32 per = (n + blockDim.x - 1) / blockDim.x;
    const u32 lo = threadIdx.x * per, hi = min(n, lo + per);
    for (u32 i = lo; i < hi; i++) v += part[i];
    v = block_sum(v, red);
    if (threadIdx.x == 0) *out = v;
}

__global__ void k_sum_grad(const double* __restrict__ gpart, u32 nedge, u32 nblk, double* __restrict__ grad) {
    pdl_wait();
    pdl_trigger();
    const u32 e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nedge) return;
    double v = 0;
    for (u32 b = 0; b < nblk; b++) v += gpart[(size_t)e * nblk + b];
    grad[e] = v;
}

// ----------------------------------------------------------- L-BFGS ----

enum { SC_GD = 0, SC_DMAX = 1, SC_SY = 2, SC_YY = 3, SC_GG = 4, SC_N = 8 };

struct Lb {
    u32 n, nCTA, Mr;  // Mr: ring slots (history + one spare)
    double *x, *g, *d, *xn, *t, *grad, *S, *Y, *rho, *gam, *sc, *part;
    u32* flags;
    int* err;
    u64 limitNs;
    double tmin, tmax;
};

// Grid reduction of three sums and one maximum, identical in every CTA:
// per-CTA partials (double-buffered by barrier parity) summed in CTA order.
__device__ bool grid_reduce(const Lb& a, double v[4], u32& epoch) {
    __shared__ double red[kLbThreads / 32][4];
    __shared__ double out[4];
    __shared__ double stage[kMaxLbCTA * 4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        double x = v[k];
        for (int o = 16; o > 0; o >>= 1) {
            const double y = __shfl_xor_sync(0xFFFFFFFFu, x, o);
            x = k == 3 ? fmax(x, y) : x + y;
        }
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][k] = x;
    }
    __syncthreads();
    const u32 par = epoch & 1u;
    if (threadIdx.x < 4) {
        double x = 0.0;
        for (u32 i = 0; i < kLbThreads / 32; i++)
            x = threadIdx.x == 3 ? fmax(x, red[i][threadIdx.x]) : x + red[i][threadIdx.x];
        a.part[((size_t)par * a.nCTA + blockIdx.x) * 4 + threadIdx.x] = x;
    }
    if (flag_barrier(a.flags, a.nCTA, blockIdx.x, ++epoch, a.err, a.limitNs)) return false;
    // all CTAs' partials in one round of loads, then summed in CTA order from
    // shared memory (a chain of dependent L2 loads cost ~14 us a reduction)
    const double* pp = a.part + (size_t)par * a.nCTA * 4;
    for (u32 i = threadIdx.x; i < a.nCTA * 4; i += kLbThreads) stage[i] = __ldcg(pp + i);
    __syncthreads();
    if (threadIdx.x < 4) {
        double x = 0.0;
        for (u32 i = 0; i < a.nCTA; i++) {
            const double y = stage[i * 4 + threadIdx.x];
            x = threadIdx.x == 3 ? fmax(x, y) : x + y;
        }
        out[threadIdx.x] = x;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; k++) v[k] = out[k];
    __syncthreads();
    return true;
}

// d = -H g by the two-loop recursion over `count` pairs starting at ring
// slot `first`; writes g.d and max|d| to sc.
__global__ void __launch_bounds__(kLbThreads) k_lb_dir(Lb a, u32 first, u32 count) {
    __shared__ double alpha[kMaxHist];
    const u32 stride = a.nCTA * kLbThreads, i0 = blockIdx.x * kLbThreads + threadIdx.x;
    u32 epoch = 0;
    for (u32 i = i0; i < a.n; i += stride) a.d[i] = a.g[i];
    for (int k = (int)count - 1; k >= 0; k--) {
        const u32 r = (first + (u32)k) % a.Mr;
        const double* s = a.S + (size_t)r * a.n;
        const double* y = a.Y + (size_t)r * a.n;
        double v[4] = {0, 0, 0, 0};
        for (u32 i = i0; i < a.n; i += stride) v[0] += s[i] * a.d[i];
        if (!grid_reduce(a, v, epoch)) return;
        const double al = a.rho[r] * v[0];
        if (threadIdx.x == 0) alpha[k] = al;
        for (u32 i = i0; i < a.n; i += stride) a.d[i] -= al * y[i];
    }
    __syncthreads();
    if (count > 0) {
        const double gm = a.gam[(first + count - 1) % a.Mr];
        for (u32 i = i0; i < a.n; i += stride) a.d[i] *= gm;
    }
    for (u32 k = 0; k < count; k++) {
        const u32 r = (first + k) % a.Mr;
        const double* s = a.S + (size_t)r * a.n;
        const double* y = a.Y + (size_t)r * a.n;
        double v[4] = {0, 0, 0, 0};
        for (u32 i = i0; i < a.n; i += stride) v[0] += y[i] * a.d[i];
        if (!grid_reduce(a, v, epoch)) return;
        const double c = alpha[k] - a.rho[r] * v[0];
        for (u32 i = i0; i < a.n; i += stride) a.d[i] += c * s[i];
    }
    double v[4] = {0, 0, 0, 0};
    for (u32 i = i0; i < a.n; i += stride) {
        const double di = -a.d[i];
        a.d[i] = di;
        v[0] += a.g[i] * di;
        v[3] = fmax(v[3], fabs(di));
    }
    if (!grid_reduce(a, v, epoch)) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.sc[SC_GD] = v[0];
        a.sc[SC_DMAX] = v[3];
    }
}

// Accept the trial point: g_new = -grad * t (gradient of -log L in log t),
// history pair into ring slot `slot`, x = xn, g = g_new.
__global__ void __launch_bounds__(kLbThreads) k_lb_accept(Lb a, u32 slot) {
    const u32 stride = a.nCTA * kLbThreads, i0 = blockIdx.x * kLbThreads + threadIdx.x;
    u32 epoch = 0;
    double v[4] = {0, 0, 0, 0};
    double* S = a.S + (size_t)slot * a.n;
    double* Y = a.Y + (size_t)slot * a.n;
    for (u32 i = i0; i < a.n; i += stride) {
        const double gn = -a.grad[i] * a.t[i];
        const double s = a.xn[i] - a.x[i], y = gn - a.g[i];
        S[i] = s;
        Y[i] = y;
        v[0] += s * y;
        v[1] += y * y;
        v[2] += gn * gn;
        a.x[i] = a.xn[i];
        a.g[i] = gn;
    }
    if (!grid_reduce(a, v, epoch)) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.sc[SC_SY] = v[0];
        a.sc[SC_YY] = v[1];
        a.sc[SC_GG] = v[2];
        a.rho[slot] = v[0] != 0.0 ? 1.0 / v[0] : 0.0;
        a.gam[slot] = v[1] > 0.0 ? v[0] / v[1] : 1.0;
    }
}

__global__ void k_lb_trial(Lb a, double step) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const double xn = a.x[i] + step * a.d[i];
    a.xn[i] = xn;
    a.t[i] = fmin(fmax(exp(xn), a.tmin), a.tmax);
}

// t <- clamp(t), x <- log t
__global__ void k_lb_init(Lb a) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const double t = fmin(fmax(a.t[i], a.tmin), a.tmax);
    a.t[i] = t;
    a.x[i] = log(t);
}

__global__ void k_lb_grad0(Lb a) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < a.n) a.g[i] = -a.grad[i] * a.t[i];
}

}  // namespace fel

using namespace fel;

// --------------------------------------------------------------- host ---

struct FelTreeHost {
    u32 ntip = 0, nn = 0, nint = 0, nedge = 0, root = 0;
    std::vector<u32> kidA, kidB, edgeA, edgeB, inOrder, outOrder;
    std::vector<u32> inOff, outOff;  // level offsets
};

static int build_tree(u32 ntip, u32 nedge, const u32* edge, FelTreeHost& T) {
    if (ntip < 2 || nedge != 2 * ntip - 2 || !edge) {
        casphy_set_last_error_msg("felsenstein: the tree must be binary with 2*ntip-2 edges");
        return CASPHY_EINVAL;
    }
    T.ntip = ntip;
    T.nedge = nedge;
    T.nn = nedge + 1;
    T.nint = ntip - 1;
    const u32 nn = T.nn, none = 0xFFFFFFFFu;
    T.kidA.assign(T.nint, none);
    T.kidB.assign(T.nint, none);
    T.edgeA.assign(T.nint, 0);
    T.edgeB.assign(T.nint, 0);
    std::vector<unsigned char> isChild(nn, 0);
    for (u32 e = 0; e < nedge; e++) {
        const u32 p = edge[2 * e], c = edge[2 * e + 1];
        if (p >= nn || c >= nn || p < ntip || isChild[c]) {
            casphy_set_last_error_msg("felsenstein: bad edge (tips must be 0..ntip-1, each node one parent)");
            return CASPHY_EINVAL;
        }
        isChild[c] = 1;
        const u32 pi = p - ntip;
        if (T.kidA[pi] == none) {
            T.kidA[pi] = c;
            T.edgeA[pi] = e;
        } else if (T.kidB[pi] == none) {
            T.kidB[pi] = c;
            T.edgeB[pi] = e;
        } else {
            casphy_set_last_error_msg("felsenstein: a node has more than two children");
            return CASPHY_EINVAL;
        }
    }
    u32 nroot = 0;
    for (u32 v = 0; v < nn; v++)
        if (!isChild[v]) {
            T.root = v;
            nroot++;
        }
    if (nroot != 1 || T.root < ntip) {
        casphy_set_last_error_msg("felsenstein: the tree needs exactly one root, an internal node");
        return CASPHY_EINVAL;
    }
    for (u32 i = 0; i < T.nint; i++)
        if (T.kidB[i] == none) {
            casphy_set_last_error_msg("felsenstein: internal nodes must have two children");
            return CASPHY_EINVAL;
        }
    // heights and depths without recursion (parents before children)
    std::vector<u32> order, height(nn, 0), depth(nn, 0);
    order.reserve(nn);
    std::vector<u32> stack{T.root};
    while (!stack.empty()) {
        const u32 v = stack.back();
        stack.pop_back();
        order.push_back(v);
        if (v >= ntip) {
            const u32 a = T.kidA[v - ntip], b = T.kidB[v - ntip];
            depth[a] = depth[b] = depth[v] + 1;
            stack.push_back(a);
            stack.push_back(b);
        }
        if (order.size() > nn) break;
    }
    if (order.size() != nn) {
        casphy_set_last_error_msg("felsenstein: the edges do not form one tree");
        return CASPHY_EINVAL;
    }
    u32 H = 0, D = 0;
    for (auto it = order.rbegin(); it != order.rend(); ++it) {
        const u32 v = *it;
        if (v >= ntip) height[v] = 1 + std::max(height[T.kidA[v - ntip]], height[T.kidB[v - ntip]]);
        H = std::max(H, height[v]);
        D = std::max(D, depth[v]);
    }
    std::vector<std::vector<u32>> byH(H + 1), byD(D + 1);
    for (u32 v = ntip; v < nn; v++) {
        byH[height[v]].push_back(v);
        byD[depth[v]].push_back(v);
    }
    T.inOff.assign(1, 0);
    for (u32 h = 1; h <= H; h++) {
        T.inOrder.insert(T.inOrder.end(), byH[h].begin(), byH[h].end());
        T.inOff.push_back((u32)T.inOrder.size());
    }
    T.outOff.assign(1, 0);
    for (u32 d = 0; d <= D; d++) {
        if (byD[d].empty()) continue;
        T.outOrder.insert(T.outOrder.end(), byD[d].begin(), byD[d].end());
        T.outOff.push_back((u32)T.outOrder.size());
    }
    return CASPHY_OK;
}

// HKY85 rate matrix in nibble order A,T,C,G (transitions A<->G, T<->C),
// scaled to one substitution per unit time; eigensystem of the symmetrised
// matrix diag(sqrt(pi)) Q diag(1/sqrt(pi)) by cyclic Jacobi rotations.
static void hky_parts(double kappa, const double* pi, Hky& m) {
    double Q[16];
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            const bool ts = (i == 0 && j == 3) || (i == 3 && j == 0) || (i == 1 && j == 2) || (i == 2 && j == 1);
            Q[i * 4 + j] = i == j ? 0.0 : pi[j] * (ts ? kappa : 1.0);
        }
    double mu = 0;
    for (int i = 0; i < 4; i++) {
        double r = 0;
        for (int j = 0; j < 4; j++) r += Q[i * 4 + j];
        Q[i * 4 + i] = -r;
        mu += pi[i] * r;
    }
    for (double& x : Q) x /= mu;
    double S[16], W[16];
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            S[i * 4 + j] = std::sqrt(pi[i]) * Q[i * 4 + j] / std::sqrt(pi[j]);
            W[i * 4 + j] = i == j ? 1.0 : 0.0;
        }
    for (int i = 0; i < 4; i++)
        for (int j = i + 1; j < 4; j++) S[i * 4 + j] = S[j * 4 + i] = 0.5 * (S[i * 4 + j] + S[j * 4 + i]);
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0;
        for (int i = 0; i < 4; i++)
            for (int j = i + 1; j < 4; j++) off += S[i * 4 + j] * S[i * 4 + j];
        if (off < 1e-32) break;
        for (int p = 0; p < 4; p++)
            for (int q = p + 1; q < 4; q++) {
                if (std::fabs(S[p * 4 + q]) < 1e-300) continue;
                const double th = (S[q * 4 + q] - S[p * 4 + p]) / (2 * S[p * 4 + q]);
                const double t = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1));
                const double c = 1 / std::sqrt(t * t + 1), s = t * c;
                for (int k = 0; k < 4; k++) {
                    const double a = S[k * 4 + p], b = S[k * 4 + q];
                    S[k * 4 + p] = c * a - s * b;
                    S[k * 4 + q] = s * a + c * b;
                }
                for (int k = 0; k < 4; k++) {
                    const double a = S[p * 4 + k], b = S[q * 4 + k];
                    S[p * 4 + k] = c * a - s * b;
                    S[q * 4 + k] = s * a + c * b;
                }
                for (int k = 0; k < 4; k++) {
                    const double a = W[k * 4 + p], b = W[k * 4 + q];
                    W[k * 4 + p] = c * a - s * b;
                    W[k * 4 + q] = s * a + c * b;
                }
            }
    }
    for (int k = 0; k < 4; k++) m.lam[k] = S[k * 4 + k];
    for (int i = 0; i < 4; i++)
        for (int k = 0; k < 4; k++) {
            m.V[i * 4 + k] = W[i * 4 + k] / std::sqrt(pi[i]);
            m.Vi[k * 4 + i] = W[i * 4 + k] * std::sqrt(pi[i]);
        }
    for (int i = 0; i < 4; i++) m.pi[i] = pi[i];
}

// One likelihood problem resident on the device, with its evaluation graphs.
struct FelProblem {
    FelTreeHost th;
    Tree T{};
    u32 nsite = 0, model = 0, W = 0, nchunk = 0, nblkTot = 0;
    Hky hky{};
    double rate = 1.0;
    double *t = nullptr, *w = nullptr, *grad = nullptr, *gpart = nullptr, *part = nullptr, *ll = nullptr;
    HkyBuf hb{};
    IrrBuf ib{};
    float *P = nullptr, *dP = nullptr;
    float2* p = nullptr;
    Lb lb{};
    cudaGraphExec_t gFull = nullptr, gLL = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    u64 launchesFull = 0, launchesLL = 0;

    ~FelProblem() {
        if (st) cudaStreamSynchronize(st);
        if (gFull) cudaGraphExecDestroy(gFull);
        if (gLL) cudaGraphExecDestroy(gLL);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (g0) cudaEventDestroy(g0);
        if (g1) cudaEventDestroy(g1);
        if (st) cudaStreamDestroy(st);
    }

    // Every kernel of an evaluation is launched with programmatic stream
    // serialisation: each begins with pdl_wait(), so stream order holds for
    // every buffer, and the next level's launch overlaps this one's tail.
    cudaError_t launchErr = cudaSuccess;
    template <class... KArgs, class... Args>
    void lp(void (*k)(KArgs...), dim3 grid, u32 block, Args... args) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = grid;
        cfg.blockDim = dim3(block);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        const cudaError_t e = cudaLaunchKernelEx(&cfg, k, args...);
        if (e != cudaSuccess && launchErr == cudaSuccess) launchErr = e;
    }

    void enqueue(bool withGrad, u64* launches) {
        u64 n = 0;
        const u32 ne = th.nedge;
        if (model == CASPHY_MODEL_HKY85) lp(k_pmat_hky, dim3((ne + 127) / 128), 128, (const double*)t, ne, hky, P, dP);
        else lp(k_pmat_irr, dim3((ne + 127) / 128), 128, (const double*)t, ne, rate, p);
        n++;
        for (u32 c = 0; c < nchunk; c++) {
            Chunk C;
            C.s0 = c * W;
            C.w = std::min(W, nsite - C.s0);
            C.W = W;
            C.nsite = nsite;
            C.blk0 = C.s0 / kSites;
            C.nblkTot = nblkTot;
            const u32 nb = (C.w + kSites - 1) / kSites;
            for (size_t lv = 0; lv + 1 < th.inOff.size(); lv++) {
                const dim3 grid(nb, th.inOff[lv + 1] - th.inOff[lv]);
                if (model == CASPHY_MODEL_HKY85) lp(k_inside_hky, grid, kSites / 2, T, hb, C, th.inOff[lv]);
                else lp(k_inside_irr, grid, kSites / 2, T, ib, C, th.inOff[lv]);
                n++;
            }
            if (model == CASPHY_MODEL_HKY85) lp(k_loglik_hky, dim3(nb), kSites, th.root, T, hb, C, hky, (const double*)w, part);
            else lp(k_loglik_irr, dim3(nb), kSites, th.root, T, ib, C, (const double*)w, part);
            n++;
            if (!withGrad) continue;
            for (size_t lv = 0; lv + 1 < th.outOff.size(); lv++) {
                const dim3 grid(nb, th.outOff[lv + 1] - th.outOff[lv]);
                if (model == CASPHY_MODEL_HKY85)
                    lp(k_outside_hky, grid, kSites / 2, th.root, T, hb, C, th.outOff[lv], hky, (const double*)w, gpart);
                else lp(k_outside_irr, grid, kSites, th.root, T, ib, C, th.outOff[lv], (const double*)w, gpart);
                n++;
            }
        }
        lp(k_sum_ll, dim3(1), 256, (const double*)part, nblkTot, ll);
        n++;
        if (withGrad) {
            lp(k_sum_grad, dim3((ne + 255) / 256), 256, (const double*)gpart, ne, nblkTot, grad);
            n++;
        }
        if (launches) *launches = n;
    }

    int capture() {
        for (int k = 0; k < 2; k++) {
            cudaGraph_t g;
            CASPHY_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            enqueue(k == 0, k == 0 ? &launchesFull : &launchesLL);
            CASPHY_CUDA_TRY(cudaStreamEndCapture(st, &g));
            if (launchErr != cudaSuccess) {
                cudaGraphDestroy(g);
                CASPHY_CUDA_TRY(launchErr);
            }
            cudaGraphExec_t ex;
            const cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
            cudaGraphDestroy(g);
            CASPHY_CUDA_TRY(e);
            (k == 0 ? gFull : gLL) = ex;
        }
        return CASPHY_OK;
    }

    // log L (and d log L / d t in `grad`) at the branch lengths in `t`:
    // eval_launch() queues the graph and the read of log L into *llOut,
    // eval_done() (after the stream is synchronised) adds its graph time
    int eval_launch(bool withGrad, double* llOut) {
        CASPHY_CUDA_TRY(cudaEventRecord(g0, st));
        CASPHY_CUDA_TRY(cudaGraphLaunch(withGrad ? gFull : gLL, st));
        CASPHY_CUDA_TRY(cudaEventRecord(g1, st));
        CASPHY_CUDA_TRY(cudaMemcpyAsync(llOut, ll, sizeof(double), cudaMemcpyDeviceToHost, st));
        return CASPHY_OK;
    }
    void eval_done() {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, g0, g1) == cudaSuccess) graphMs += ms;
    }
    int eval(bool withGrad, double* llOut) {
        if (int rc = eval_launch(withGrad, llOut)) return rc;
        CASPHY_CUDA_TRY(cudaStreamSynchronize(st));
        eval_done();
        return CASPHY_OK;
    }
    cudaEvent_t g0 = nullptr, g1 = nullptr;
    double graphMs = 0;
};

static int setup_problem(FelProblem& F, DeviceScope& ds, u32 ntip, u32 nedge, const u32* edge, const double* brlen,
                         u32 nsite, const u32* codes, const double* weights, const casphy_felsenstein_model* model,
                         u32 hist) {
    if (!brlen || !codes || !model || nsite == 0) return CASPHY_EINVAL;
    int rc = build_tree(ntip, nedge, edge, F.th);
    if (rc) return rc;
    F.nsite = nsite;
    F.model = model->model;
    const bool isH = F.model == CASPHY_MODEL_HKY85;
    if (!isH && F.model != CASPHY_MODEL_IRREVERSIBLE) {
        casphy_set_last_error_msg("felsenstein: unknown model");
        return CASPHY_EINVAL;
    }
    for (u32 e = 0; e < nedge; e++)
        if (!(brlen[e] >= 0.0) || !std::isfinite(brlen[e])) {
            casphy_set_last_error_msg("felsenstein: branch lengths must be finite and >= 0");
            return CASPHY_EINVAL;
        }
    if (weights)
        for (u32 s = 0; s < nsite; s++)
            if (!(weights[s] >= 0.0) || !std::isfinite(weights[s])) {
                casphy_set_last_error_msg("felsenstein: site weights must be finite and >= 0");
                return CASPHY_EINVAL;
            }
    if (isH) {
        double s = 0;
        for (int i = 0; i < 4; i++) {
            if (!(model->pi[i] > 0) || !std::isfinite(model->pi[i])) {
                casphy_set_last_error_msg("felsenstein: HKY85 base frequencies must be > 0");
                return CASPHY_EINVAL;
            }
            s += model->pi[i];
        }
        if (!(model->kappa > 0) || !std::isfinite(model->kappa)) {
            casphy_set_last_error_msg("felsenstein: HKY85 kappa must be > 0");
            return CASPHY_EINVAL;
        }
        double pi[4];
        for (int i = 0; i < 4; i++) pi[i] = model->pi[i] / s;
        hky_parts(model->kappa, pi, F.hky);
    } else {
        if (!(model->rate > 0) || !std::isfinite(model->rate) || model->nallele == 0 || model->nallele > 0x7FF0u) {
            casphy_set_last_error_msg("felsenstein: irreversible model needs rate > 0 and 1 <= nallele <= 32752");
            return CASPHY_EINVAL;
        }
        for (size_t i = 0; i < (size_t)ntip * nsite; i++)
            if (codes[i] > model->nallele + 1) {
                casphy_set_last_error_msg("felsenstein: tip code beyond nallele + 1");
                return CASPHY_ERANGE;
            }
    }
    F.rate = model->rate;
    const u32 nint = F.th.nint;
    // site chunk width: a multiple of the block size whose partials fit the budget
    const u64 perSite = (u64)nint * (isH ? 36u : 32u);
    const u32 full = (nsite + kSites - 1) / kSites * kSites;
    u64 Wb = full;
    if (model->mem_budget) Wb = std::max<u64>(kSites, model->mem_budget / perSite / kSites * kSites);
    F.W = (u32)std::min<u64>(Wb, full);
    F.nchunk = (nsite + F.W - 1) / F.W;
    F.nblkTot = (nsite + kSites - 1) / kSites;
    const u32 qstride = isH ? 1 : model->nallele + 1;
    int nsm = 148;
    {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    }
    const u32 nCTA = (u32)std::max(1, std::min(nsm, (int)kMaxLbCTA)), Mr = hist + 1;
    if (hist >= kMaxHist) return CASPHY_EINVAL;
    struct Bufs {
        u32 *kidA, *kidB, *edgeA, *edgeB, *inO, *outO, *codes, *flags, *inEB, *outEB;
        uint4 *inInfo, *outInfo;
        double *t, *w, *grad, *gpart, *part, *ll;
        double *x, *g, *d, *xn, *S, *Y, *rho, *gam, *sc, *lpart;
        float *P, *dP, *q;
        float2* p;
        float4 *L, *U;
        int* E;
        int* err;
    };
    const size_t nv = hist ? nedge : 0;
    auto lay = [&](Carve& c) {
        Bufs b;
        b.kidA = c.take<u32>(nint);
        b.kidB = c.take<u32>(nint);
        b.edgeA = c.take<u32>(nint);
        b.edgeB = c.take<u32>(nint);
        b.inO = c.take<u32>(nint);
        b.outO = c.take<u32>(nint);
        b.inInfo = c.take<uint4>(nint);
        b.outInfo = c.take<uint4>(nint);
        b.inEB = c.take<u32>(nint);
        b.outEB = c.take<u32>(nint);
        b.codes = c.take<u32>((size_t)ntip * nsite);
        b.flags = c.take<u32>(16 * nCTA);
        b.err = c.take<int>(1);
        b.t = c.take<double>(nedge);
        b.w = c.take<double>(nsite);
        b.grad = c.take<double>(nedge);
        b.gpart = c.take<double>((size_t)nedge * F.nblkTot);
        b.part = c.take<double>(F.nblkTot);
        b.ll = c.take<double>(1);
        b.x = c.take<double>(nv);
        b.g = c.take<double>(nv);
        b.d = c.take<double>(nv);
        b.xn = c.take<double>(nv);
        b.S = c.take<double>(Mr * nv);
        b.Y = c.take<double>(Mr * nv);
        b.rho = c.take<double>(Mr);
        b.gam = c.take<double>(Mr);
        b.sc = c.take<double>(SC_N);
        b.lpart = c.take<double>(8 * (size_t)nCTA);
        b.P = c.take<float>(isH ? 16 * (size_t)nedge : 0);
        b.dP = c.take<float>(isH ? 16 * (size_t)nedge : 0);
        b.p = c.take<float2>(isH ? 0 : nedge);
        b.q = c.take<float>(isH ? 0 : (size_t)nsite * qstride);
        b.L = c.take<float4>((size_t)nint * F.W);
        b.U = c.take<float4>((size_t)nint * F.W);
        b.E = c.take<int>(isH ? (size_t)nint * F.W : 0);
        return b;
    };
    Carve cv;
    lay(cv);
    void* base = nullptr;
    rc = ds.reserve(cv.off + 256, &base);
    if (rc) return rc;
    Carve c2;
    c2.base = static_cast<char*>(base);
    const Bufs L = lay(c2);
    CASPHY_CUDA_TRY(cudaStreamCreateWithFlags(&F.st, cudaStreamNonBlocking));
    CASPHY_CUDA_TRY(cudaEventCreate(&F.e0));
    CASPHY_CUDA_TRY(cudaEventCreate(&F.e1));
    CASPHY_CUDA_TRY(cudaEventCreate(&F.g0));
    CASPHY_CUDA_TRY(cudaEventCreate(&F.g1));
    cudaStream_t st = F.st;
    auto up = [&](void* d, const void* h, size_t n) { return cudaMemcpyAsync(d, h, n, cudaMemcpyHostToDevice, st); };
    CASPHY_CUDA_TRY(up(L.kidA, F.th.kidA.data(), 4ull * nint));
    CASPHY_CUDA_TRY(up(L.kidB, F.th.kidB.data(), 4ull * nint));
    CASPHY_CUDA_TRY(up(L.edgeA, F.th.edgeA.data(), 4ull * nint));
    CASPHY_CUDA_TRY(up(L.edgeB, F.th.edgeB.data(), 4ull * nint));
    CASPHY_CUDA_TRY(up(L.inO, F.th.inOrder.data(), 4ull * F.th.inOrder.size()));
    CASPHY_CUDA_TRY(up(L.outO, F.th.outOrder.data(), 4ull * F.th.outOrder.size()));
    // node, children and edges per level position, so a block finds its node's
    // whole neighbourhood with one dependent load
    std::vector<uint4> inInfo(nint), outInfo(nint);
    std::vector<u32> inEB(nint), outEB(nint);
    for (u32 i = 0; i < nint; i++) {
        const u32 a = F.th.inOrder[i] - ntip, b = F.th.outOrder[i] - ntip;
        inInfo[i] = make_uint4(F.th.inOrder[i], F.th.kidA[a], F.th.kidB[a], F.th.edgeA[a]);
        inEB[i] = F.th.edgeB[a];
        outInfo[i] = make_uint4(F.th.outOrder[i], F.th.kidA[b], F.th.kidB[b], F.th.edgeA[b]);
        outEB[i] = F.th.edgeB[b];
    }
    CASPHY_CUDA_TRY(up(L.inInfo, inInfo.data(), sizeof(uint4) * nint));
    CASPHY_CUDA_TRY(up(L.outInfo, outInfo.data(), sizeof(uint4) * nint));
    CASPHY_CUDA_TRY(up(L.inEB, inEB.data(), 4ull * nint));
    CASPHY_CUDA_TRY(up(L.outEB, outEB.data(), 4ull * nint));
    CASPHY_CUDA_TRY(up(L.codes, codes, 4ull * ntip * nsite));
    CASPHY_CUDA_TRY(up(L.t, brlen, 8ull * nedge));
    std::vector<double> wv(nsite, 1.0);
    if (weights) wv.assign(weights, weights + nsite);
    CASPHY_CUDA_TRY(up(L.w, wv.data(), 8ull * nsite));
    CASPHY_CUDA_TRY(cudaMemsetAsync(L.err, 0, sizeof(int), st));
    std::vector<float> q;
    if (!isH) {
        // allele frequencies per site: given, or the tips' allele counts
        q.assign((size_t)nsite * qstride, 0.f);
        std::vector<double> cnt(qstride);
        for (u32 s = 0; s < nsite; s++) {
            std::fill(cnt.begin(), cnt.end(), 0.0);
            if (model->allele_freq) {
                for (u32 a = 1; a < qstride; a++) cnt[a] = std::max(0.0, model->allele_freq[(size_t)s * qstride + a]);
            } else {
                for (u32 i = 0; i < ntip; i++) {
                    const u32 c = codes[(size_t)i * nsite + s];
                    if (c >= 2) cnt[c - 1] += 1;
                }
            }
            double tot = 0;
            for (u32 a = 1; a < qstride; a++) tot += cnt[a];
            for (u32 a = 1; a < qstride; a++)
                q[(size_t)s * qstride + a] = tot > 0 ? (float)(cnt[a] / tot) : (float)(1.0 / (qstride - 1));
        }
        CASPHY_CUDA_TRY(up(L.q, q.data(), 4 * q.size()));
    }
    F.T = Tree{ntip, L.kidA, L.kidB, L.edgeA, L.edgeB, L.inO, L.outO, L.inInfo, L.inEB, L.outInfo, L.outEB};
    F.t = L.t;
    F.w = L.w;
    F.grad = L.grad;
    F.gpart = L.gpart;
    F.part = L.part;
    F.ll = L.ll;
    F.hb = HkyBuf{L.codes, L.L, L.E, L.U, L.P, L.dP};
    F.ib = IrrBuf{L.codes, L.L, L.U, L.p, L.q, qstride, (float)model->rate};
    F.P = L.P;
    F.dP = L.dP;
    F.p = L.p;
    F.lb = Lb{nedge, nCTA, Mr, L.x, L.g, L.d, L.xn, L.t, L.grad, L.S, L.Y, L.rho, L.gam, L.sc, L.lpart,
              L.flags, L.err, 5ull * 1000 * 1000 * 1000, 1e-8, 10.0};
    rc = F.capture();
    if (rc) return rc;
    // host staging buffers (wv, q) must outlive the copies
    CASPHY_CUDA_TRY(cudaStreamSynchronize(st));
    return CASPHY_OK;
}

static int lb_coop(FelProblem& F, const void* fn, void** args) {
    CASPHY_CUDA_TRY(cudaMemsetAsync(F.lb.flags, 0, sizeof(u32) * 16 * F.lb.nCTA, F.st));
    CASPHY_CUDA_TRY(cudaLaunchCooperativeKernel(fn, dim3(F.lb.nCTA), dim3(kLbThreads), args, 0, F.st));
    return CASPHY_OK;
}

// Reads `n` doubles from the device scalars at `src` together with the grid
// barrier's error flag, with one synchronisation.
static int lb_read(FelProblem& F, const double* src, double* dst, size_t n) {
    int err = 0;
    CASPHY_CUDA_TRY(cudaMemcpyAsync(&err, F.lb.err, sizeof(int), cudaMemcpyDeviceToHost, F.st));
    CASPHY_CUDA_TRY(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToHost, F.st));
    CASPHY_CUDA_TRY(cudaStreamSynchronize(F.st));
    if (err) {
        casphy_set_last_error_msg("felsenstein: a grid barrier of the L-BFGS step timed out");
        return CASPHY_ETIMEOUT;
    }
    return CASPHY_OK;
}

// Per-edge central differences of log L into F.grad (as d log L / d t).
// The step is taken in x = log t: t e^{+-h} with h = 1e-3, large enough that
// the binary32 rounding of the partials (about 1e-7 of |log L|) stays well
// below the difference, small enough that the O(h^2) truncation does too.
static int fd_gradient(FelProblem& F, casphy_blopt_stats& st) {
    const u32 n = F.th.nedge;
    const double h = 1e-3;
    std::vector<double> t(n), g(n);
    CASPHY_CUDA_TRY(cudaMemcpyAsync(t.data(), F.t, 8ull * n, cudaMemcpyDeviceToHost, F.st));
    CASPHY_CUDA_TRY(cudaStreamSynchronize(F.st));
    for (u32 i = 0; i < n; i++) {
        const double tp = t[i] * std::exp(h), tm = t[i] * std::exp(-h);
        double lp = 0, lm = 0;
        int rc;
        CASPHY_CUDA_TRY(cudaMemcpyAsync(F.t + i, &tp, 8, cudaMemcpyHostToDevice, F.st));
        if ((rc = F.eval(false, &lp))) return rc;
        CASPHY_CUDA_TRY(cudaMemcpyAsync(F.t + i, &tm, 8, cudaMemcpyHostToDevice, F.st));
        if ((rc = F.eval(false, &lm))) return rc;
        CASPHY_CUDA_TRY(cudaMemcpyAsync(F.t + i, &t[i], 8, cudaMemcpyHostToDevice, F.st));
        st.evaluations += 2;
        g[i] = (lp - lm) / (2 * h) / t[i];
    }
    CASPHY_CUDA_TRY(cudaMemcpyAsync(F.grad, g.data(), 8ull * n, cudaMemcpyHostToDevice, F.st));
    CASPHY_CUDA_TRY(cudaStreamSynchronize(F.st));
    return CASPHY_OK;
}

}  // namespace casphy

extern "C" int casphy_felsenstein_loglik(uint32_t ntip, uint32_t nedge, const uint32_t* edge, const double* brlen,
                                         uint32_t nsite, const uint32_t* tip_codes, const double* site_weights,
                                         const casphy_felsenstein_model* model, double* loglik, double* grad) {
    using namespace casphy;
    int rc = require_device();
    if (rc) return rc;
    if (!loglik) return CASPHY_EINVAL;
    DeviceScope ds;
    FelProblem F;
    rc = setup_problem(F, ds, ntip, nedge, edge, brlen, nsite, tip_codes, site_weights, model, 0);
    if (rc) return rc;
    rc = F.eval(grad != nullptr, loglik);
    if (rc) return rc;
    if (grad) {
        CASPHY_CUDA_TRY(cudaMemcpyAsync(grad, F.grad, sizeof(double) * nedge, cudaMemcpyDeviceToHost, F.st));
        CASPHY_CUDA_TRY(cudaStreamSynchronize(F.st));
    }
    return CASPHY_OK;
}

extern "C" int casphy_felsenstein_optimize(uint32_t ntip, uint32_t nedge, const uint32_t* edge, double* brlen,
                                           uint32_t nsite, const uint32_t* tip_codes, const double* site_weights,
                                           const casphy_felsenstein_model* model, int gradient_mode,
                                           uint32_t max_iter, double rel_tol, casphy_blopt_stats* stats) {
    using namespace casphy;
    int rc = require_device();
    if (rc) return rc;
    if (gradient_mode != CASPHY_GRAD_ADJOINT && gradient_mode != CASPHY_GRAD_CENTRAL_DIFF) return CASPHY_EINVAL;
    const u32 M = 8;
    DeviceScope ds;
    FelProblem F;
    rc = setup_problem(F, ds, ntip, nedge, edge, brlen, nsite, tip_codes, site_weights, model, M);
    if (rc) return rc;
    const bool adj = gradient_mode == CASPHY_GRAD_ADJOINT;
    const bool trace = std::getenv("CASPHY_TRACE") != nullptr;
    const u32 n = nedge, nb = (n + 255) / 256;
    casphy_blopt_stats st{};
    Lb a = F.lb;
    CASPHY_CUDA_TRY(cudaEventRecord(F.e0, F.st));
    k_lb_init<<<nb, 256, 0, F.st>>>(a);
    // objective f = -log L at the start, and its gradient in x = log t
    double ll = 0;
    if ((rc = F.eval(adj, &ll))) return rc;
    st.evaluations++;
    if (!adj && (rc = fd_gradient(F, st))) return rc;
    k_lb_grad0<<<nb, 256, 0, F.st>>>(a);
    st.loglik_start = ll;
    double f = -ll;
    u32 first = 0, count = 0, quiet = 0;
    const u32 kQuiet = 5;
    // After an accepted point that does not end the run, the accept, the next
    // direction (with the history the accept gives when s.y > 1e-12), its
    // unit-step trial and that trial's evaluation are queued together and
    // read with one synchronisation.  These are the launches the step-by-step
    // sequence makes when s.y > 1e-12 and the direction descends; otherwise
    // the direction and the trial are discarded and made again by that
    // sequence.  The kernels are deterministic, so the iterates are the same
    // either way; a discarded evaluation still counts in `evaluations`.
    bool spec = false;
    double specGd = 0, specDmax = 0, specLl = 0;
    for (u32 it = 0; it < max_iter; it++) {
        double gd = specGd, dmax = specDmax;
        if (!spec) {
            u32 cnt = count;
            double sc[2] = {0, 0};
            for (int attempt = 0; attempt < 2; attempt++) {
                void* args[] = {&a, &first, &cnt};
                if ((rc = lb_coop(F, (const void*)k_lb_dir, args))) return rc;
                if ((rc = lb_read(F, a.sc + SC_GD, sc, 2))) return rc;
                if (sc[0] < 0 || cnt == 0) break;
                cnt = 0;  // not a descent direction: restart from steepest descent
            }
            if (cnt == 0 && count != 0) first = (first + count) % a.Mr;
            count = cnt;
            gd = sc[0];
            dmax = sc[1];
            if (!(gd < 0)) break;  // stationary
        }
        double step = count == 0 ? std::min(1.0, 1.0 / std::max(dmax, 1e-12)) : 1.0;
        double fn = 0;
        bool accepted = false;
        for (int ls = 0; ls < 40; ls++) {
            if (ls == 0 && spec) {
                ll = specLl;  // the speculated unit step (count > 0, so step is 1)
            } else {
                k_lb_trial<<<nb, 256, 0, F.st>>>(a, step);
                if ((rc = F.eval(adj, &ll))) return rc;
                st.evaluations++;
            }
            fn = -ll;
            if (fn <= f + 1e-4 * step * gd) {
                accepted = true;
                break;
            }
            step *= 0.5;
        }
        spec = false;
        if (!accepted) {
            // leave t at the accepted point x
            k_lb_trial<<<nb, 256, 0, F.st>>>(a, 0.0);
            break;
        }
        if (!adj && (rc = fd_gradient(F, st))) return rc;
        // converged when log L has changed by at most rel_tol (relative) in
        // each of the last kQuiet steps: one short step alone does not stop
        const double rel = std::fabs(f - fn) / std::max(std::fabs(f), 1e-300);
        const u32 quietNext = rel <= rel_tol ? quiet + 1 : 0;
        u32 slot = (first + count) % a.Mr;
        void* args[] = {&a, &slot};
        if ((rc = lb_coop(F, (const void*)k_lb_accept, args))) return rc;
        double sy = 0;
        if (adj && quietNext < kQuiet && it + 1 < max_iter) {
            u32 cntN = count < M ? count + 1 : count, firstN = count < M ? first : (first + 1) % a.Mr;
            void* dargs[] = {&a, &firstN, &cntN};
            if ((rc = lb_coop(F, (const void*)k_lb_dir, dargs))) return rc;
            k_lb_trial<<<nb, 256, 0, F.st>>>(a, 1.0);
            if ((rc = F.eval_launch(adj, &specLl))) return rc;
            double sc3[3] = {0, 0, 0};  // g.d, max|d| of the direction; s.y of the accept
            if ((rc = lb_read(F, a.sc + SC_GD, sc3, 3))) return rc;
            F.eval_done();
            st.evaluations++;
            sy = sc3[SC_SY - SC_GD];
            specGd = sc3[SC_GD - SC_GD];
            specDmax = sc3[SC_DMAX - SC_GD];
            spec = sy > 1e-12 && specGd < 0;
        } else {
            if ((rc = lb_read(F, a.sc + SC_SY, &sy, 1))) return rc;
        }
        st.iterations++;
        if (sy > 1e-12) {
            if (count < M) count++;
            else first = (first + 1) % a.Mr;
        }
        if (trace)
            std::fprintf(stderr, "blopt it %u f %.10f df %.3e gd %.3e step %.3e hist %u sy %.3e%s\n", it, fn, fn - f,
                         gd, step, count, sy, spec || !(adj && quietNext < kQuiet && it + 1 < max_iter) ? "" : " (speculated step discarded)");
        f = fn;
        quiet = quietNext;
        if (quiet >= kQuiet) break;
    }
    CASPHY_CUDA_TRY(cudaEventRecord(F.e1, F.st));
    CASPHY_CUDA_TRY(cudaEventSynchronize(F.e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, F.e0, F.e1);
    std::vector<double> t(n);
    CASPHY_CUDA_TRY(cudaMemcpyAsync(t.data(), a.t, 8ull * n, cudaMemcpyDeviceToHost, F.st));
    CASPHY_CUDA_TRY(cudaStreamSynchronize(F.st));
    for (u32 i = 0; i < n; i++) brlen[i] = t[i];
    st.loglik_end = -f;
    st.seconds = ms / 1e3;
    st.site_chunks = F.nchunk;
    st.levels_inside = (u32)F.th.inOff.size() - 1;
    st.levels_outside = (u32)F.th.outOff.size() - 1;
    st.launches_per_eval = adj ? F.launchesFull : F.launchesLL;
    st.eval_seconds = F.graphMs / 1e3;
    if (stats) *stats = st;
    return CASPHY_OK;
}
