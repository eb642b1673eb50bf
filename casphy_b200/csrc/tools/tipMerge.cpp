// Drop-in for `tipMerge <prefix> <pShared>` (cu/tipMerge.cu:130-461):
// <prefix>.nNeighbor + <prefix>.idx (radiusNeighbor outputs) -> <prefix>.member
// (one category per line).
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
    const double pShared = atof(argv[2]);
    uint32_t d0 = 0, ntip = 0;
    std::vector<uint32_t> counts;
    if (!tool::read_mat(prefix + ".nNeighbor", d0, ntip, counts)) {
        printf("No nNeighbor input.\n");
        return 0;
    }
    counts.resize(ntip);
    uint64_t total = 0;
    for (uint32_t c : counts) total += c;
    std::vector<uint32_t> idx(total ? total : 1, 0u);
    FILE* f = fopen((prefix + ".idx").c_str(), "rb");
    if (!f) {
        printf("No indices input.\n");
        return 0;
    }
    const size_t got = fread(idx.data(), sizeof(uint32_t), total, f);
    fclose(f);
    (void)got;  // a short file leaves zeros, like the reference's unchecked fread
    if (dev < 0) return tool::fail("tipMerge", CASPHY_ENODEV);
    std::vector<int32_t> member(ntip ? ntip : 1);
    const int rc = casphy_tip_merge(ntip, counts.data(), idx.data(), pShared, member.data());
    if (rc == CASPHY_ERANGE) {
        printf("%s\n", casphy_last_error());
        return 0;
    }
    if (rc) return tool::fail("tipMerge", rc);
    FILE* out = fopen((prefix + ".member").c_str(), "w");
    if (!out) return 1;
    for (uint32_t i = 0; i < ntip; i++) fprintf(out, "%d\n", member[i]);
    fclose(out);
    printf("tipMerge: %.2fs elapsed for %u tips.\n", tool::now_s() - t0, ntip);
    return 0;
}
