#include "toolio.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <unistd.h>

#include "casphy.h"

namespace tool {

bool read_header(const std::string& path, uint32_t& d0, uint32_t& d1) {
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) return false;
    uint32_t dim[2] = {0, 0};
    size_t r = fread(dim, sizeof(uint32_t), 2, f);
    fclose(f);
    d0 = dim[0];
    d1 = dim[1];
    return r == 2;
}

bool read_mat(const std::string& path, uint32_t& d0, uint32_t& d1, std::vector<uint32_t>& data) {
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) return false;
    uint32_t dim[2] = {0, 0};
    if (fread(dim, sizeof(uint32_t), 2, f) != 2) dim[0] = dim[1] = 0;
    d0 = dim[0];
    d1 = dim[1];
    data.assign((size_t)d0 * d1, 0u);
    if (!data.empty()) {
        size_t got = fread(data.data(), sizeof(uint32_t), data.size(), f);
        (void)got;
    }
    fclose(f);
    return true;
}

bool read_f64(const std::string& path, size_t n, std::vector<double>& out) {
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) return false;
    out.assign(n, 0.0);
    if (n) {
        size_t got = fread(out.data(), sizeof(double), n, f);
        (void)got;
    }
    fclose(f);
    return true;
}

bool write_raw(const std::string& path, const void* data, size_t bytes, bool append) {
    FILE* f = fopen(path.c_str(), append ? "ab" : "wb");
    if (!f) return false;
    bool ok = bytes == 0 || fwrite(data, 1, bytes, f) == bytes;
    return fclose(f) == 0 && ok;
}

bool write_mat(const std::string& path, uint32_t d0, uint32_t d1, const uint32_t* data, size_t n) {
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) return false;
    uint32_t dim[2] = {d0, d1};
    bool ok = fwrite(dim, sizeof(uint32_t), 2, f) == 2;
    if (n) ok = ok && fwrite(data, sizeof(uint32_t), n, f) == n;
    return fclose(f) == 0 && ok;
}

int pick_device() {
    const int n = casphy_device_count();
    if (n <= 0) return -1;
    const char* env = getenv("CASPHY_DEVICE");
    int dev;
    if (env && *env) {
        dev = atoi(env) % n;
    } else {
        srand((unsigned)time(nullptr) ^ (unsigned)getpid());
        dev = rand() % n;
    }
    return casphy_set_device(dev) == CASPHY_OK ? dev : -1;
}

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

int fail(const char* tool, int status) {
    fprintf(stderr, "%s: %s (%s)\n", tool, casphy_strerror(status), casphy_last_error());
    return 1;
}

}  // namespace tool
