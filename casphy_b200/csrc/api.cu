// Library-wide C ABI helpers: status strings, last-error text, the per-device
// workspace arena, and device selection.
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "runtime.h"

static thread_local char g_last_error[512] = "";

void casphy_set_last_cuda_error(cudaError_t e, const char* what, const char* file, int line) {
    snprintf(g_last_error, sizeof(g_last_error), "%s:%d %s -> %s (%s)", file, line, what,
             cudaGetErrorName(e), cudaGetErrorString(e));
}
void casphy_set_last_error_msg(const char* msg) {
    snprintf(g_last_error, sizeof(g_last_error), "%s", msg);
}

extern "C" int casphy_abi_version(void) { return CASPHY_ABI_VERSION; }

extern "C" const char* casphy_last_error(void) { return g_last_error; }

extern "C" int casphy_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

extern "C" int casphy_set_device(int device) {
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        casphy_set_last_cuda_error(e, "cudaSetDevice", __FILE__, __LINE__);
        return CASPHY_ECUDA;
    }
    return CASPHY_OK;
}

extern "C" const char* casphy_strerror(int s) {
    switch (s) {
        case CASPHY_OK: return "ok";
        case CASPHY_EINVAL: return "invalid argument";
        case CASPHY_ERANGE: return "value out of supported range";
        case CASPHY_ENOMEM: return "out of memory";
        case CASPHY_ECUDA: return "CUDA runtime error";
        case CASPHY_ETIMEOUT: return "device-side wait timed out";
        case CASPHY_EIO: return "input/output error";
        case CASPHY_ENODEV: return "no CUDA device";
        case CASPHY_EINTERNAL: return "internal error";
        default: return "unknown status";
    }
}

namespace casphy {

// Grow-only device arena per device.  Calls hold the device's lock for their
// whole duration, so one process runs one hot-path call per GPU at a time;
// separate processes (the R fork-cluster pattern) each have their own arena.
struct Arena {
    std::mutex mu;
    void* base = nullptr;
    size_t cap = 0;
    void* aux = nullptr;  // second grow-only block for outputs sized mid-call
    size_t auxCap = 0;
};
static std::mutex g_arenas_mu;
static std::vector<Arena*> g_arenas;

static Arena* arena_for(int dev) {
    std::lock_guard<std::mutex> g(g_arenas_mu);
    if ((int)g_arenas.size() <= dev) g_arenas.resize(dev + 1, nullptr);
    if (!g_arenas[dev]) g_arenas[dev] = new Arena();
    return g_arenas[dev];
}

DeviceScope::DeviceScope() {
    cudaGetDevice(&dev);
    arena = arena_for(dev);
    static_cast<Arena*>(arena)->mu.lock();
}
DeviceScope::~DeviceScope() { static_cast<Arena*>(arena)->mu.unlock(); }

// Grow-only block: a bigger request frees the old block and allocates
// 1/8 more than asked (or exactly the request when that fails).
static int grow(void** base, size_t* cap, size_t bytes, const char* what) {
    if (bytes > *cap) {
        if (*base) cudaFree(*base);
        *base = nullptr;
        *cap = 0;
        size_t want = bytes + (bytes >> 3);
        cudaError_t e = cudaMalloc(base, want);
        if (e != cudaSuccess) {
            cudaGetLastError();
            e = cudaMalloc(base, bytes);
            want = bytes;
        }
        if (e != cudaSuccess) {
            cudaGetLastError();
            *base = nullptr;
            casphy_set_last_cuda_error(e, what, __FILE__, __LINE__);
            return CASPHY_ENOMEM;
        }
        *cap = want;
    }
    return CASPHY_OK;
}

int DeviceScope::reserve(size_t bytes, void** out) {
    Arena* a = static_cast<Arena*>(arena);
    const int rc = grow(&a->base, &a->cap, bytes, "cudaMalloc(arena)");
    if (rc) return rc;
    *out = a->base;
    return CASPHY_OK;
}

int DeviceScope::reserve_aux(size_t bytes, void** out) {
    Arena* a = static_cast<Arena*>(arena);
    const int rc = grow(&a->aux, &a->auxCap, bytes, "cudaMalloc(aux)");
    if (rc) return rc;
    *out = a->aux;
    return CASPHY_OK;
}

int require_device() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        casphy_set_last_error_msg("no CUDA device visible");
        return CASPHY_ENODEV;
    }
    return CASPHY_OK;
}

}  // namespace casphy
