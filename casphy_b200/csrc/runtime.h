// Host-side runtime pieces shared by the entry points: the per-device
// workspace arena (one lock per device held for a whole call) and a bump
// allocator that carves typed, 256-byte aligned buffers out of it.
#pragma once
#include <cstddef>
#include <cstdint>

namespace casphy {

struct DeviceScope {
    int dev = 0;
    void* arena = nullptr;
    DeviceScope();
    ~DeviceScope();
    // Returns a device block of at least `bytes`, valid until the scope ends.
    // A later reserve() in the same scope may move the block.
    int reserve(size_t bytes, void** out);
    // A second block, independent of reserve()'s, for outputs whose size is
    // only known part-way through a call.
    int reserve_aux(size_t bytes, void** out);
};

struct Carve {
    size_t off = 0;
    char* base = nullptr;
    template <class T>
    T* take(size_t n) {
        off = (off + 255) & ~size_t(255);
        T* p = reinterpret_cast<T*>(base ? base + off : nullptr);
        off += n * sizeof(T);
        return p;
    }
};

int require_device();

}  // namespace casphy
