// Drop-in for `tryRadius <prefix> <radius> <nReplicate>` (cu/tryRadius.cu:
// 52-189): counts neighbours of nReplicate rows drawn with rand() % ntip after
// srand(time), like the reference; <prefix>.nNeighbor = {2, n} + rows + counts.
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
        return argc < 3 ? 0 : 1;
    }
    const int dev = tool::pick_device();
    const int32_t radius = atoi(argv[2]);
    const uint32_t nrep = (uint32_t)atoi(argv[3]);
    const std::string prefix = argv[1];
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
    if (dev < 0) return tool::fail("tryRadius", CASPHY_ENODEV);
    if (ntip == 0) return tool::fail("tryRadius", CASPHY_EINVAL);
    std::vector<uint32_t> q(nrep), counts(nrep);
    std::srand((unsigned)std::time(nullptr));
    for (uint32_t i = 0; i < nrep; i++) q[i] = (uint32_t)(std::rand() % ntip);
    int rc = casphy_try_radius_bit(nrow, ntip, bmat.data(), w.data(), radius, nrep, q.data(), counts.data());
    if (rc) return tool::fail("tryRadius", rc);
    std::vector<uint32_t> body(q);
    body.insert(body.end(), counts.begin(), counts.end());
    if (!tool::write_mat(prefix + ".nNeighbor", 2, nrep, body.data(), body.size())) return 1;
    printf("\nradiusNeighbor: %.2fs elapsed for %u tips.\n", tool::now_s() - t0, ntip);
    return 0;
}
