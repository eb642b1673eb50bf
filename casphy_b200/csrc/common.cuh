// Shared device helpers for the CasPhy sm_100a kernels.
//
// Everything here is plain CUDA C++/inline PTX for sm_100a: cache-hinted
// loads for data other CTAs write during a persistent launch, a grid barrier
// whose wait is bounded by %globaltimer (it records CASPHY_ETIMEOUT and
// returns instead of spinning forever), and order-preserving integer keys
// for the (score, node) argmax the greedy joins use.
#pragma once
#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "../../include/casphy.h"

typedef uint32_t u32;
typedef uint16_t u16;
typedef uint64_t u64;

#define CASPHY_CUDA_TRY(expr)                                  \
    do {                                                      \
        cudaError_t _e = (expr);                              \
        if (_e != cudaSuccess) {                              \
            casphy_set_last_cuda_error(_e, #expr, __FILE__, __LINE__); \
            return CASPHY_ECUDA;                              \
        }                                                     \
    } while (0)

// Records the last CUDA failure for casphy_last_error(); defined in api.cu.
void casphy_set_last_cuda_error(cudaError_t e, const char* what, const char* file, int line);
void casphy_set_last_error_msg(const char* msg);

// ---------------------------------------------------------------------------
// Programmatic dependent launch, for chains of kernels in one stream or graph
// that are launched with cudaLaunchAttributeProgrammaticStreamSerialization.
// pdl_wait() returns once the preceding kernel has completed and its writes
// are visible (at once for a kernel launched without the attribute);
// pdl_trigger() lets the next kernel begin launching once every CTA of this
// one has issued it or exited.  A kernel that calls pdl_wait() before it
// touches global memory keeps plain stream order for every buffer, and the
// next kernel's launch overlaps this one's tail.

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// ---------------------------------------------------------------------------
// loads/stores that bypass L1 (data written by other CTAs of a live grid)

__device__ __forceinline__ u32 ld_cg_u32(const u32* p) {
    u32 v;
    asm volatile("ld.global.cg.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ u64 ld_cg_u64(const u64* p) {
    u64 v;
    asm volatile("ld.global.cg.u64 %0, [%1];" : "=l"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ uint4 ld_cg_v4(const void* p) {
    uint4 v;
    asm volatile("ld.global.cg.v4.u32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p));
    return v;
}
// Asynchronous 16-byte global -> shared copy through L2 only (cp.async.cg);
// both addresses 16-byte aligned.  cp_async_wait_all() waits for this
// thread's copies; a block barrier after it publishes them to the block.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const u32 sa = static_cast<u32>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// Closes this thread's copies issued so far into a group; cp_async_wait_group<N>
// waits until at most N of its groups are still in flight.
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ u16 ld_cg_u16(const u16* p) {
    u16 v;
    asm volatile("ld.global.cg.u16 %0, [%1];" : "=h"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ u32 ld_acquire_u32(const u32* p) {
    u32 v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(u32* p, u32 v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ u64 globaltimer_ns() {
    u64 t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// All-to-all flag barrier for nCTA co-resident CTAs: CTA `self` (its index
// among them) publishes `epoch` in its own flag; threads 0..nCTA-1 each wait
// for one CTA's flag.  Every wait gives up after limit_ns and records
// CASPHY_ETIMEOUT.
__device__ __forceinline__ int flag_barrier(u32* flags, u32 nCTA, u32 self, u32 epoch, int* err, u64 limit_ns) {
    __syncthreads();
    if (nCTA == 1) return 0;  // one CTA: the block barrier orders its global accesses
    if (threadIdx.x == 0) st_release_u32(flags + self * 16u, epoch);  // gpu-scope release, cumulative
    int fail = 0;
    if (threadIdx.x < nCTA) {
        const u32* f = flags + threadIdx.x * 16u;
        if (ld_acquire_u32(f) < epoch) {
            const u64 t0 = globaltimer_ns();
            while (ld_acquire_u32(f) < epoch) {
                if (*(volatile int*)err) { fail = 1; break; }
                if (globaltimer_ns() - t0 > limit_ns) {
                    atomicCAS(err, 0, CASPHY_ETIMEOUT);
                    fail = 1;
                    break;
                }
                __nanosleep(32);
            }
        }
    }
    return __syncthreads_or(fail);
}

// ---------------------------------------------------------------------------
// Grid barrier for a cooperatively launched grid (all CTAs co-resident).
// The wait gives up after `limit_ns`, records CASPHY_ETIMEOUT in *err and
// returns non-zero; any CTA that sees *err set also returns non-zero.

struct GridSync {
    u32 count;
    u32 gen;
    int err;
    u32 pad;
};

__device__ __forceinline__ int grid_barrier(GridSync* gs, u32 nblocks, u64 limit_ns) {
    __shared__ int s_fail;
    __syncthreads();
    if (threadIdx.x == 0) {
        int fail = 0;
        u32 g = ld_acquire_u32(&gs->gen);
        __threadfence();
        u32 arrived = atomicAdd(&gs->count, 1u);
        if (arrived == nblocks - 1) {
            atomicExch(&gs->count, 0u);
            __threadfence();
            st_release_u32(&gs->gen, g + 1u);
        } else {
            u64 t0 = globaltimer_ns();
            u32 ns = 32;
            while (ld_acquire_u32(&gs->gen) == g) {
                if (*(volatile int*)&gs->err) { fail = 1; break; }
                if (globaltimer_ns() - t0 > limit_ns) {
                    atomicCAS(&gs->err, 0, CASPHY_ETIMEOUT);
                    fail = 1;
                    break;
                }
                __nanosleep(ns);
                if (ns < 256) ns <<= 1;
            }
        }
        if (*(volatile int*)&gs->err) fail = 1;
        s_fail = fail;
    }
    __syncthreads();
    return s_fail;
}

// ---------------------------------------------------------------------------
// Order-preserving keys.  A join candidate is (value, node); the reference
// argmax prefers the larger value, then the smaller node index, and starts
// from (-1, 0) (cu/joinEdgeIndel.cu:110-121).  key = ord(value) << 32 | ~node
// turns that into an unsigned max.  -0 is folded onto +0 so equal values tie.

__device__ __host__ __forceinline__ u32 ord_f32(float f) {
    u32 b;
#ifdef __CUDA_ARCH__
    b = __float_as_uint(f);
#else
    __builtin_memcpy(&b, &f, 4);
#endif
    if (b == 0x80000000u) b = 0u;
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __host__ __forceinline__ u32 ord_f16(u16 h) {
    if (h == 0x8000u) h = 0u;
    u32 b = h;
    return (b & 0x8000u) ? (~b & 0xFFFFu) : (b | 0x8000u);
}
__device__ __host__ __forceinline__ bool is_nan_f16(u16 h) { return (h & 0x7C00u) == 0x7C00u && (h & 0x3FFu); }
__device__ __host__ __forceinline__ bool is_nan_f32_bits(u32 b) { return (b & 0x7F800000u) == 0x7F800000u && (b & 0x7FFFFFu); }

#define ORD_F16_NEG1 0x43FFu      // ord_f16(0xBC00)
#define ORD_F32_NEG1 0x407FFFFFu  // ord_f32(-1.0f)

__device__ __forceinline__ u64 make_key(u32 ordv, u32 node) { return ((u64)ordv << 32) | (u64)(~node); }
__device__ __forceinline__ u32 key_node(u64 k) { return ~(u32)k; }
__device__ __forceinline__ u32 key_ord(u64 k) { return (u32)(k >> 32); }

__device__ __forceinline__ u64 warp_max_u64(u64 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        u64 w = __shfl_xor_sync(0xFFFFFFFFu, v, o);
        v = w > v ? w : v;
    }
    return v;
}

// Block-wide max of a u64 (blockDim.x a multiple of 32, <= 1024).
__device__ __forceinline__ u64 block_max_u64(u64 v, u64* scratch /* >= 32 */) {
    v = warp_max_u64(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) scratch[wid] = v;
    __syncthreads();
    const int nw = blockDim.x >> 5;
    v = lane < nw ? scratch[lane] : 0ull;
    v = warp_max_u64(v);
    __syncthreads();
    return v;
}
