// Drop-in for `tryRadiusDNA <prefix> <radius> <nReplicate>` (cu/tryRadiusDNA.cu:
// 76-178): rows drawn with rand() % ntip after srand(time), like the reference.
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <string>
#include <vector>

#include "casphy.h"
#include "toolio.h"

int main(int argc, char* argv[]) {
    setbuf(stdout, nullptr);
    const double t0 = tool::now_s();
    if (argc < 4) {
        printf("Error: no sufficient args.\n");
        return 0;
    }
    const uint32_t radius = (uint32_t)atoi(argv[2]);
    const uint32_t nrep = (uint32_t)atoi(argv[3]);
    const std::string prefix = argv[1];
    const int dev = tool::pick_device();
    uint32_t ntip = 0, nbinRaw = 0;
    std::vector<uint32_t> raw;
    if (!tool::read_mat(prefix + ".tbmat", ntip, nbinRaw, raw)) {
        printf("No bmat input.\n");
        return 0;
    }
    if (dev < 0) return tool::fail("tryRadiusDNA", CASPHY_ENODEV);
    if (ntip == 0) return tool::fail("tryRadiusDNA", CASPHY_EINVAL);
    std::vector<uint32_t> q(nrep), counts(nrep);
    std::srand((unsigned)std::time(nullptr));
    for (uint32_t i = 0; i < nrep; i++) q[i] = (uint32_t)(std::rand() % ntip);
    int rc = casphy_try_radius_dna(ntip, nbinRaw, raw.data(), radius, nrep, q.data(), counts.data());
    if (rc) return tool::fail("tryRadiusDNA", rc);
    float avg = 0;
    for (uint32_t i = 0; i < nrep; i++) avg += counts[i];
    avg /= nrep;
    printf("Average nNeighbor: %.2f\n", avg);
    std::vector<uint32_t> body(q);
    body.insert(body.end(), counts.begin(), counts.end());
    if (!tool::write_mat(prefix + ".nNeighbor", 2, nrep, body.data(), body.size())) return 1;
    printf("radiusNeighborDNA: %.2fs elapsed for %u tips.\n", tool::now_s() - t0, ntip);
    return 0;
}
