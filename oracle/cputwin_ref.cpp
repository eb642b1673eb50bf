// C wrapper around the reference's CPU implementations of the hot path (the
// functions R calls when no CUDA path is given): greedyJoinEdge2 and
// greedyJoinEdgeBitReverse (src/functions.cpp:1880-2017, :3316-3461, called by
// phy.join, R/CasPhy_functions.R:1621-1649) and the per-row radius functions
// radiusWeightedParallel / radiusWeightedDNAParallel (:1825-1857, :4021-4036,
// applied over rows by parSapply in R/CasPhy_functions.R:160-200, :1729).
// The ref build recipe pastes those functions and their helpers in front of
// this file from src/functions.cpp.  Test infrastructure only: the timed CPU
// baseline beside the B200 path, never part of the product.
#include <omp.h>

#include <cstdint>
#include <cstring>

// mat: nsite x ntip column-major (R's t(regularize.mat(mat, mat))): -1 missing,
// 0 unedited, 1.. alleles.  weight: nstate x nsite column-major.  edge_out
// (optional): (3 + nsite) x (2 ntip - 1) column-major, the function's result.
extern "C" int ref_greedy_join_edge2(uint32_t ntip, uint32_t nsite, const int32_t* mat, uint32_t nstate,
                                     const double* weight, const int32_t* tipSize, int minSize, float minRatio,
                                     int32_t* edge_out) {
    Rcpp::IntegerMatrix m((int)nsite, (int)ntip);
    std::memcpy(m.data(), mat, sizeof(int32_t) * (size_t)ntip * nsite);
    Rcpp::NumericMatrix w((int)nstate, (int)nsite);
    std::memcpy(w.data(), weight, sizeof(double) * (size_t)nstate * nsite);
    Rcpp::IntegerVector ts((int)ntip);
    for (uint32_t i = 0; i < ntip; i++) ts(i) = tipSize ? tipSize[i] : 1;
    Rcpp::IntegerMatrix e = greedyJoinEdge2(m, w, ts, minSize, minRatio, false);
    if (edge_out) std::memcpy(edge_out, e.data(), sizeof(int32_t) * (size_t)e.nrow() * e.ncol());
    r_alloc_release();
    return 0;
}

// mat: nbin x ntip column-major words (bit b of word x = site 32 x + b);
// weight: 32 nbin per-site weights.  edge_out (optional): 2 x (2 ntip - 2).
extern "C" int ref_greedy_join_edge_bit_reverse(uint32_t ntip, uint32_t nbin, const uint32_t* mat,
                                                const double* weight, int ancestralType, int32_t* edge_out) {
    Rcpp::IntegerMatrix m((int)nbin, (int)ntip);
    std::memcpy(m.data(), mat, sizeof(uint32_t) * (size_t)ntip * nbin);
    Rcpp::NumericVector w((int)nbin * 32);
    std::memcpy(w.data(), weight, sizeof(double) * (size_t)nbin * 32);
    Rcpp::List out = greedyJoinEdgeBitReverse(m, w, false, ancestralType);
    for (auto& x : out.mats)
        if (x.first == "edge" && edge_out)
            std::memcpy(edge_out, x.second.data(), sizeof(int32_t) * 2 * (size_t)(2 * ntip - 2));
    r_alloc_release();
    return 0;
}

// Rows [row0, row1) of radiusWeightedParallel over mat (ncell x nword
// column-major, one row per cell), one row per call as R's parSapply does,
// spread over nthreads threads (R's fork cluster of ncore workers).  Each
// thread holds its own weight vector, as each forked worker does.  out:
// (row1 - row0) x (nbin + 1), nbin = ceil(ncell / 32): the count then the
// neighbour bitmap of each row.
extern "C" int ref_radius_weighted_rows(uint32_t ncell, uint32_t nword, const uint32_t* mat, int maxChar,
                                        const double* weight, float radius, uint32_t row0, uint32_t row1,
                                        int nthreads, uint32_t* out) {
    Rcpp::IntegerMatrix m((int)ncell, (int)nword);
    std::memcpy(m.data(), mat, sizeof(uint32_t) * (size_t)ncell * nword);
    const size_t nb1 = ((ncell + 31) / 32) + 1;
#pragma omp parallel num_threads(nthreads)
    {
        Rcpp::NumericVector w((int)nword * 32);
        std::memcpy(w.data(), weight, sizeof(double) * (size_t)nword * 32);
        Rcpp::IntegerMatrix mt = m;
#pragma omp for schedule(dynamic, 16)
        for (long r = (long)row0; r < (long)row1; r++) {
            Rcpp::IntegerVector o = radiusWeightedParallel((int)r, mt, maxChar, w, radius);
            std::memcpy(out + (size_t)(r - row0) * nb1, o.data(), sizeof(uint32_t) * nb1);
        }
    }
    return 0;
}

// Rows [row0, row1) of radiusWeightedDNAParallel over mat (nint x nseq
// column-major: the fasta2bin rows, four columns per int, one code byte
// each); weight: 4 nint per-column weights.  Threads and out as above,
// nbin = ceil(nseq / 32).
extern "C" int ref_radius_weighted_dna_rows(uint32_t nseq, uint32_t nint, const uint32_t* mat, const double* weight,
                                            float radius, uint32_t row0, uint32_t row1, int nthreads,
                                            uint32_t* out) {
    Rcpp::IntegerMatrix m((int)nint, (int)nseq);
    std::memcpy(m.data(), mat, sizeof(uint32_t) * (size_t)nseq * nint);
    const size_t nb1 = ((nseq + 31) / 32) + 1;
#pragma omp parallel num_threads(nthreads)
    {
        Rcpp::NumericVector w((int)nint * 4);
        std::memcpy(w.data(), weight, sizeof(double) * (size_t)nint * 4);
        Rcpp::IntegerMatrix mt = m;
#pragma omp for schedule(dynamic, 16)
        for (long r = (long)row0; r < (long)row1; r++) {
            Rcpp::IntegerVector o = radiusWeightedDNAParallel((int)r, mt, w, radius);
            std::memcpy(out + (size_t)(r - row0) * nb1, o.data(), sizeof(uint32_t) * nb1);
        }
    }
    return 0;
}

// approximateCompare2_AVX2 (src/functions.cpp:5450-5600) for one query tree.
// clade: the reference tree's clade matrix as nodeDesBig writes it without
// header (nbin x (nnode1 - 1) column-major, column k = node ntip+nnode1-1-k,
// 0-based).  edge1, edge2: 1-based (parent, child) pairs in ape's cladewise
// order.  ref2qry: nnode1 x 2 column-major (node, distance); qry2ref:
// nnode2 x 3 column-major (node, distance, size).  Returns 1 when the
// function ran out of cache (it returns 0 to R then), else 0.
static int approx_compare_one(uint32_t ntip, uint32_t nnode1, uint32_t nbin, int32_t* clade, const Rcpp::IntegerMatrix& e1,
                              uint32_t nedge2, const int32_t* edge2, uint32_t nnode2, int cacheSize, float threshold,
                              int32_t* ref2qry, int32_t* qry2ref) {
    BigMatrix bm;
    bm.nr = nbin;
    bm.nc = nnode1 - 1;
    bm.d = clade;
    Rcpp::IntegerMatrix e2((int)nedge2, 2);
    for (uint32_t i = 0; i < nedge2; i++) {
        e2(i, 0) = edge2[2 * i];
        e2(i, 1) = edge2[2 * i + 1];
    }
    Rcpp::List out = approximateCompare2_AVX2(static_cast<SEXP>(&bm), (int)ntip, e1, e2, (int)nnode2, cacheSize,
                                              threshold);
    if (out.null) return 1;
    for (auto& x : out.mats) {
        if (x.first == "ref2qry" && ref2qry) std::memcpy(ref2qry, x.second.data(), sizeof(int32_t) * 2 * (size_t)nnode1);
        if (x.first == "qry2ref" && qry2ref) std::memcpy(qry2ref, x.second.data(), sizeof(int32_t) * 3 * (size_t)nnode2);
    }
    return 0;
}

static Rcpp::IntegerMatrix edge_matrix(uint32_t nedge, const int32_t* edge) {
    Rcpp::IntegerMatrix e((int)nedge, 2);
    for (uint32_t i = 0; i < nedge; i++) {
        e(i, 0) = edge[2 * i];
        e(i, 1) = edge[2 * i + 1];
    }
    return e;
}

extern "C" int ref_approx_compare(uint32_t ntip, uint32_t nnode1, uint32_t nbin, int32_t* clade, uint32_t nedge1,
                                  const int32_t* edge1, uint32_t nedge2, const int32_t* edge2, uint32_t nnode2,
                                  int cacheSize, float threshold, int32_t* ref2qry, int32_t* qry2ref) {
    return approx_compare_one(ntip, nnode1, nbin, clade, edge_matrix(nedge1, edge1), nedge2, edge2, nnode2,
                              cacheSize, threshold, ref2qry, qry2ref);
}

// The query trees of cal.abs / clade.support (R/bootstrap_functions.R:34-57,
// :190-202), spread over nthreads threads as parLapply spreads them over a
// fork cluster.  Tree t: edges2 + 2 off2[t], nedge2[t] edges, nnode2[t]
// internal nodes; outputs at ref2qry + 2 nnode1 t and qry2ref + 3 qoff[t].
// Returns the number of trees that ran out of cache.
extern "C" int ref_approx_compare_many(uint32_t ntip, uint32_t nnode1, uint32_t nbin, int32_t* clade,
                                       uint32_t nedge1, const int32_t* edge1, uint32_t ntree, const uint64_t* off2,
                                       const uint32_t* nedge2, const int32_t* edges2, const uint32_t* nnode2,
                                       const uint64_t* qoff, int cacheSize, float threshold, int nthreads,
                                       int32_t* ref2qry, int32_t* qry2ref) {
    int bad = 0;
#pragma omp parallel num_threads(nthreads) reduction(+ : bad)
    {
        const Rcpp::IntegerMatrix e1 = edge_matrix(nedge1, edge1);
#pragma omp for schedule(dynamic, 1)
        for (long t = 0; t < (long)ntree; t++)
            bad += approx_compare_one(ntip, nnode1, nbin, clade, e1, nedge2[t], edges2 + 2 * off2[t], nnode2[t],
                                      cacheSize, threshold, ref2qry + 2 * (size_t)nnode1 * t,
                                      qry2ref ? qry2ref + 3 * qoff[t] : nullptr);
    }
    return bad;
}
