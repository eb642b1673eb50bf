// Drop-in for `Felsenstein <prefix> <seed>` (cu/Felsenstein.cu:68-151), the
// bootstrap column resampler: draws nbin*4 byte positions with
// std::mt19937(seed) and std::uniform_int_distribution<uint32_t>(0,
// nbin*4-1) -- the same library draws as the reference's host code -- sorts
// them, and writes <prefix>B<seed>.idx ({1, nbin*4} + positions) and
// <prefix>B<seed>.bin (the gathered rows, gathered on the GPU).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <string>
#include <vector>

#include "casphy.h"
#include "toolio.h"

int main(int argc, char* argv[]) {
    setbuf(stdout, nullptr);
    const double t0 = tool::now_s();
    if (argc < 3) {
        printf("Error: no sufficient args.\n");
        return 0;
    }
    const uint32_t seed = (uint32_t)atoi(argv[2]);
    char tag[24];
    snprintf(tag, sizeof(tag), "B%d", (int)seed);
    const std::string prefix = argv[1];
    uint32_t ntip = 0, nbin = 0;
    std::vector<uint32_t> in;
    if (!tool::read_mat(prefix + ".bin", ntip, nbin, in)) {
        printf("No input.\n");
        return 0;
    }
    const int dev = tool::pick_device();
    if (dev < 0) return tool::fail("Felsenstein", CASPHY_ENODEV);
    const uint32_t n = nbin * 4;
    std::vector<uint32_t> idx(n);
    std::mt19937 gen(seed);
    std::uniform_int_distribution<uint32_t> dist(0, n - 1);
    for (uint32_t i = 0; i < n; i++) idx[i] = dist(gen);
    std::sort(idx.begin(), idx.end());
    if (!tool::write_mat(prefix + tag + ".idx", 1, n, idx.data(), n)) return 1;
    std::vector<uint32_t> out((size_t)ntip * nbin);
    int rc = casphy_resample_columns(ntip, nbin, in.data(), n, idx.data(), out.data());
    if (rc) return tool::fail("Felsenstein", rc);
    if (!tool::write_mat(prefix + tag + ".bin", ntip, nbin, out.data(), out.size())) return 1;
    printf("Felsenstein sampling: %.2fs elapsed for %u tips.\n", tool::now_s() - t0, ntip);
    return 0;
}
