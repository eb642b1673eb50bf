// Drop-in for `nodeKeepBit <prefix> <cutoff>` (cu/nodeKeepBit.cu): reads
// <prefix>.nodeState2, <prefix>.edge2 and <prefix>.tboutmat, writes the kept
// node ids to <prefix>.retainNode, one per line.
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
        printf("usage: nodeKeepBit <prefix> <cutoff>\n");
        return 1;
    }
    const int dev = tool::pick_device();
    const std::string prefix = argv[1];
    const uint32_t cutoff = (uint32_t)atoi(argv[2]);
    uint32_t nnode = 0, ncol = 0, nedge = 0, two = 0, nRetain = 0, ocol = 0;
    std::vector<uint32_t> state, edge, outmat;
    if (!tool::read_mat(prefix + ".nodeState2", nnode, ncol, state)) {
        printf("No nodeState input.\n");
        return 0;
    }
    if (!tool::read_mat(prefix + ".edge2", nedge, two, edge)) {
        printf("No edge input.\n");
        return 0;
    }
    edge.resize((size_t)nedge * 2, 0u);
    if (!tool::read_header(prefix + ".tboutmat", nRetain, ocol)) {
        FILE* f = fopen((prefix + ".tboutmat").c_str(), "rb");
        if (!f) {
            printf("No outmat input.\n");
            return 0;
        }
        fclose(f);
    }
    {
        // the reference reads nRetain rows of ncol values (ncol from the state file)
        FILE* f = fopen((prefix + ".tboutmat").c_str(), "rb");
        uint32_t dim[2] = {0, 0};
        if (fread(dim, sizeof(uint32_t), 2, f) != 2) dim[0] = 0;
        nRetain = dim[0];
        outmat.assign((size_t)nRetain * ncol, 0u);
        if (!outmat.empty()) {
            size_t got = fread(outmat.data(), sizeof(uint32_t), outmat.size(), f);
            (void)got;
        }
        fclose(f);
    }
    if (dev < 0) return tool::fail("nodeKeepBit", CASPHY_ENODEV);
    std::vector<uint32_t> kept(nedge ? nedge : 1);
    uint32_t nkept = 0;
    int rc = casphy_node_keep_bit(nnode, ncol, state.data(), nedge, edge.data(), nRetain, outmat.data(), cutoff,
                                     kept.data(), &nkept);
    if (rc) return tool::fail("nodeKeepBit", rc);
    FILE* out = fopen((prefix + ".retainNode").c_str(), "w");
    if (!out) return 1;
    for (uint32_t i = 0; i < nkept; i++) fprintf(out, "%u\n", kept[i]);
    fclose(out);
    printf("nodeKeepBit: %.2fs elapsed for %u nodes and %u outgroups in GPU %d.\\n", tool::now_s() - t0, nnode, nRetain, dev);
    return 0;
}
