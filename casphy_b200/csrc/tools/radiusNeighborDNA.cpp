#include <algorithm>
// Drop-in for `radiusNeighborDNA <prefix> <radius>` (cu/radiusNeighborDNA.cu:
// 111-380): <prefix>.tbmat (fasta2bin codes) -> <prefix>.idx, <prefix>.nNeighbor.
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
    const uint32_t radius = (uint32_t)atoi(argv[2]);
    printf("%u devices detected\n", (unsigned)casphy_device_count());
    const int dev = tool::pick_device();
    const std::string prefix = argv[1];
    uint32_t ntip = 0, nbinRaw = 0;
    std::vector<uint32_t> raw;
    if (!tool::read_mat(prefix + ".tbmat", ntip, nbinRaw, raw)) {
        printf("No bmat input.\n");
        return 0;
    }
    if (dev < 0) return tool::fail("radiusNeighborDNA", CASPHY_ENODEV);
    std::vector<uint32_t> counts(ntip);
    uint64_t total = 0;
    // one search: the library allocates the lists at their counted size
    uint32_t* lists = nullptr;
    const int rc = casphy_radius_dna_lists(ntip, nbinRaw, raw.data(), radius, counts.data(), &lists, &total);
    if (rc) return tool::fail("radiusNeighborDNA", rc);
    const bool ok = tool::write_raw(prefix + ".idx", lists, sizeof(uint32_t) * total) &&
                    tool::write_mat(prefix + ".nNeighbor", 1, ntip, counts.data(), ntip);
    casphy_free(lists);
    if (!ok) return 1;
    printf("radiusNeighborDNA: %.2fs elapsed for %u tips.\n", tool::now_s() - t0, ntip);
    return 0;
}
