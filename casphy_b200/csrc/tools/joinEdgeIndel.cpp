// Drop-in for `joinEdgeIndel <prefix> <wfile> <nState> <minSize> <minRatio>`
// (cu/joinEdgeIndel.cu:244-578): reads <prefix>.tbmat, <wfile> (nState x ncol
// float64) and <prefix>.tipSize, writes <prefix>.edge2 and
// <prefix>.nodeState2 with the same bytes, on the GPU through libcasphy.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "casphy.h"
#include "toolio.h"

int main(int argc, char* argv[]) {
    setbuf(stdout, nullptr);
    const double t0 = tool::now_s();
    if (argc < 6) {
        printf("usage: joinEdgeIndel <prefix> <wfile> <nState> <minSize> <minRatio>\n");
        return 1;
    }
    const int dev = tool::pick_device();
    const std::string prefix = argv[1];
    const uint32_t nState = (uint32_t)atoi(argv[3]);
    const uint32_t minSize = (uint32_t)atoi(argv[4]);
    const float minRatio = (float)atof(argv[5]);
    uint32_t ntip = 0, ncol = 0;
    std::vector<uint32_t> codes;
    if (!tool::read_mat(prefix + ".tbmat", ntip, ncol, codes)) {
        printf("No tbmat input.\n");
        return 0;
    }
    std::vector<double> w;
    if (!tool::read_f64(argv[2], (size_t)ncol * nState, w)) {
        printf("No weight input.\n");
        return 0;
    }
    uint32_t d0 = 0, d1 = 0;
    std::vector<uint32_t> tipSize;
    if (!tool::read_mat(prefix + ".tipSize", d0, d1, tipSize)) {
        printf("No tipSize input.\n");
        return 0;
    }
    tipSize.resize(ntip, 0u);
    if (dev < 0) return tool::fail("joinEdgeIndel", CASPHY_ENODEV);
    const uint32_t nedge = ntip ? 2 * ntip - 2 : 0;
    const uint32_t nrows = ntip > 1 ? ntip - 1 : 1;
    std::vector<uint32_t> edge((size_t)nedge * 2 + 2), state((size_t)nrows * ncol);
    casphy_join_stats st;
    int rc = casphy_join_indel(ntip, ncol, codes.data(), nState, w.data(), tipSize.data(), minSize, minRatio,
                               edge.data(), state.data(), &st);
    if (rc) return tool::fail("joinEdgeIndel", rc);
    if (!tool::write_mat(prefix + ".edge2", nedge, 2, edge.data(), (size_t)nedge * 2) ||
        !tool::write_mat(prefix + ".nodeState2", ntip - 1, ncol, state.data(), (size_t)nrows * ncol)) {
        fprintf(stderr, "joinEdgeIndel: cannot write outputs for %s\n", prefix.c_str());
        return 1;
    }
    printf("joinEdgeIndel: %.2fs elapsed for %u tips in GPU %d.\n", tool::now_s() - t0, ntip, dev);
    return 0;
}
