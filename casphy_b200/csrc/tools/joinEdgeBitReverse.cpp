// Drop-in for `joinEdgeBitReverse <prefix> <wfile> <ancestralType>`
// (cu/joinEdgeBitReverse.cu:285-615): <prefix>.tbmat + <wfile> (nbin*32
// float64) -> <prefix>.edge2 and <prefix>.nodeState2.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "casphy.h"
#include "toolio.h"

int main(int argc, char* argv[]) {
    setbuf(stdout, nullptr);
    const double t0 = tool::now_s();
    if (argc < 4) {
        printf("usage: joinEdgeBitReverse <prefix> <wfile> <ancestralType>\n");
        return 1;
    }
    const int dev = tool::pick_device();
    const std::string prefix = argv[1];
    const int ancestralType = atoi(argv[3]);
    uint32_t ntip = 0, nbin = 0;
    std::vector<uint32_t> words;
    if (!tool::read_mat(prefix + ".tbmat", ntip, nbin, words)) {
        printf("No tbmat input.\n");
        return 0;
    }
    std::vector<double> w;
    if (!tool::read_f64(argv[2], (size_t)nbin * 32, w)) {
        printf("No weight input.\n");
        return 0;
    }
    if (dev < 0) return tool::fail("joinEdgeBitReverse", CASPHY_ENODEV);
    const uint32_t nedge = ntip ? 2 * ntip - 2 : 0, nrows = ntip > 1 ? ntip - 1 : 1;
    std::vector<uint32_t> edge((size_t)nedge * 2 + 2), state((size_t)nrows * nbin);
    int rc = casphy_join_bit(ntip, nbin, words.data(), w.data(), ancestralType, edge.data(), state.data(), nullptr);
    if (rc) return tool::fail("joinEdgeBitReverse", rc);
    if (!tool::write_mat(prefix + ".edge2", nedge, 2, edge.data(), (size_t)nedge * 2) ||
        !tool::write_mat(prefix + ".nodeState2", ntip - 1, nbin, state.data(), (size_t)nrows * nbin)) {
        fprintf(stderr, "joinEdgeBitReverse: cannot write outputs for %s\n", prefix.c_str());
        return 1;
    }
    printf("joinEdgeBit: %.2fs elapsed for %u tips in GPU %d.\n", tool::now_s() - t0, ntip, dev);
    return 0;
}
