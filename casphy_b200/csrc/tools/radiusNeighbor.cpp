#include <algorithm>
// Drop-in for `radiusNeighbor <prefix> <radius>` (cu/radiusNeighbor.cu:162-470):
// <prefix>.bmat (word-plane-major bits) + <prefix>.w -> <prefix>.idx and
// <prefix>.nNeighbor.
#include <cstdio>
#include <cstdlib>
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
    printf("%u devices detected\n", (unsigned)casphy_device_count());
    const int dev = tool::pick_device();
    const std::string prefix = argv[1];
    const int32_t radius = atoi(argv[2]);
    uint32_t nrow = 0, ntip = 0;
    std::vector<uint32_t> bmat;
    if (!tool::read_mat(prefix + ".bmat", nrow, ntip, bmat)) {
        printf("No bmat input.\n");
        return 0;
    }
    std::vector<double> w;
    if (!tool::read_f64(prefix + ".w", (size_t)nrow * 32, w)) {
        printf("No weight input.\n");
        return 0;
    }
    if (dev < 0) return tool::fail("radiusNeighbor", CASPHY_ENODEV);
    std::vector<uint32_t> counts(ntip);
    uint64_t total = 0;
    // one search: the library allocates the lists at their counted size
    uint32_t* lists = nullptr;
    const int rc = casphy_radius_bit_lists(nrow, ntip, bmat.data(), w.data(), radius, counts.data(), &lists, &total);
    if (rc) return tool::fail("radiusNeighbor", rc);
    const bool ok = tool::write_raw(prefix + ".idx", lists, sizeof(uint32_t) * total) &&
                    tool::write_mat(prefix + ".nNeighbor", 1, ntip, counts.data(), ntip);
    casphy_free(lists);
    if (!ok) return 1;
    printf("radiusNeighbor: %.2fs elapsed for %u tips.\n", tool::now_s() - t0, ntip);
    return 0;
}
