// C wrapper around the reference's CPU functions (ancestralBitReverse,
// charAncestralEC, nodeDesBig), which the ref build recipe pastes in front of
// this file from src/functions.cpp.  Test infrastructure only: it produces the golden
// outputs the oracle restatement and the GPU path are checked against.
#include <cstdint>
#include <cstring>

extern "C" int ref_ancestral_bit(uint32_t ntip, uint32_t nnode, uint32_t nbin, const uint32_t* mat, uint32_t nedge,
                                 const uint32_t* edge, uint32_t* state, uint32_t* len) {
    Rcpp::IntegerMatrix m((int)nbin, (int)ntip), e((int)nedge, 2);
    std::memcpy(m.data(), mat, sizeof(uint32_t) * (size_t)ntip * nbin);
    for (uint32_t i = 0; i < nedge; i++) {
        e(i, 0) = (int)edge[2 * i] + 1;
        e(i, 1) = (int)edge[2 * i + 1] + 1;
    }
    Rcpp::List out = ancestralBitReverse(m, e, (int)ntip, (int)nnode);
    for (auto& x : out.mats)
        if (x.first == "nodeState") std::memcpy(state, x.second.data(), sizeof(uint32_t) * (size_t)nnode * nbin);
    for (auto& x : out.vecs)
        if (x.first == "edgeLen") std::memcpy(len, x.second.data(), sizeof(uint32_t) * nedge);
    return 0;
}

extern "C" int ref_ancestral_char(uint32_t ntip, uint32_t nnode, uint32_t nsite, const int32_t* mat, uint32_t nedge,
                                  const uint32_t* edge, const uint32_t* tipSize, float minSize, float minRatio,
                                  int32_t* state, uint32_t* len) {
    Rcpp::IntegerMatrix m((int)nsite, (int)ntip), e((int)nedge, 2);
    std::memcpy(m.data(), mat, sizeof(int32_t) * (size_t)ntip * nsite);
    for (uint32_t i = 0; i < nedge; i++) {
        e(i, 0) = (int)edge[2 * i] + 1;
        e(i, 1) = (int)edge[2 * i + 1] + 1;
    }
    Rcpp::IntegerVector ts((int)ntip);
    for (uint32_t i = 0; i < ntip; i++) ts(i) = (int)tipSize[i];
    Rcpp::List out = charAncestralEC(m, e, ts, (int)nnode, minSize, minRatio);
    for (auto& x : out.mats)
        if (x.first == "nodeState") std::memcpy(state, x.second.data(), sizeof(int32_t) * (size_t)nnode * nsite);
    for (auto& x : out.vecs)
        if (x.first == "edgeLen") std::memcpy(len, x.second.data(), sizeof(uint32_t) * nedge);
    return 0;
}

// nodeDesBig writes the clade rows to a file (header {nnode-1, nbin} when
// header is true) and returns the internal node sizes.
extern "C" int ref_node_des_big(uint32_t ntip, uint32_t nnode, uint32_t nedge, const uint32_t* edge,
                                const char* path, int header, int32_t* sizes_out) {
    Rcpp::IntegerMatrix e((int)nedge, 2);
    for (uint32_t i = 0; i < nedge; i++) {
        e(i, 0) = (int)edge[2 * i] + 1;
        e(i, 1) = (int)edge[2 * i + 1] + 1;
    }
    Rcpp::IntegerVector out = nodeDesBig(e, (int)nnode, (int)ntip, std::string(path), 8192, header != 0);
    for (int i = 0; i < out.size(); i++) sizes_out[i] = out(i);
    r_alloc_release();
    return out.size();
}
