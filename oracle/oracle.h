/*
 * CPU oracle for the CasPhy tree-building hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library or the drop-in
 * executables links this code.  It is loaded by tests/, by
 * __graft_entry__.smoke() as the checker, and by bench.py's cpu_baseline /
 * --impl reference leg as the timed CPU restatement ("port") of the
 * reference algorithm.
 *
 * Every function restates the HOST + KERNEL semantics of one reference
 * executable (file:line cited at each definition in oracle.c), including its
 * arithmetic type (binary16 sums for the indel join, binary32 sums for the
 * bit join and bit radius search) and its tie-breaking rules, so outputs are
 * byte-identical to what the reference writes on the same inputs.
 *
 * Status codes: 0 ok, otherwise one of the CASPHY_E* values in
 * include/casphy.h (mirrored here so the oracle builds standalone).
 */
#ifndef CASPHY_ORACLE_H
#define CASPHY_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_OK 0
#define ORACLE_EINVAL 1
#define ORACLE_ERANGE 2
#define ORACLE_ENOMEM 3
#define ORACLE_EINTERNAL 9

/* Non-zero forces joinEdgeIndel's binary16 emulation even when an exact
 * integer sum would give the same values. */
extern int oracle_force_f16;
/* Non-zero selects the indel join's column-scan engine (integer weights
 * only; same outputs, for trees of 10^5 cells). */
extern int oracle_indel_colscan;

/* binary16 helpers (exposed for unit tests) */
uint16_t oracle_f64_to_f16(double x);
double oracle_f16_to_f64(uint16_t h);
uint16_t oracle_f16_add(uint16_t a, uint16_t b);

/* joinEdgeIndel.  codes: ntip x ncol row-major (0 missing, 1 unedited, >=2
 * allele).  w: nState x ncol doubles (index (code-2)*ncol + site).
 * Outputs: edge_out 2*(2*ntip-2) u32 (pre-order relabelled), state_out
 * max(ntip-1,1) x ncol u32 (root first).  stats (nullable): [0] stale
 * recomputes, [1] pair-scores evaluated, [2] joins. */
int oracle_join_indel(uint32_t ntip, uint32_t ncol, const uint32_t *codes,
                      uint32_t nState, const double *w, const uint32_t *tipSize,
                      uint32_t minSize, float minRatio, uint32_t *edge_out,
                      uint32_t *state_out, uint64_t *stats, int nthreads);

/* The same join in phases (test infrastructure for a parallel engine): up to
 * maxBatch stale rescans per phase, and with pairJoins a second join in a
 * phase when it is provably the sequential loop's next decision.  Same
 * outputs as oracle_join_indel; stats (nullable): [0] stale rescans, [1]
 * pair-scores, [2] joins, [3] phases, [4] phases with two joins, [5] pairs
 * given up because a table of each of tableCTAs ranges' top two records
 * could not vouch for them (tableCTAs 0: every record is visible). */
int oracle_join_indel_phased(uint32_t ntip, uint32_t ncol, const uint32_t *codes, uint32_t nState,
                             const double *w, const uint32_t *tipSize, uint32_t minSize, float minRatio,
                             uint32_t maxBatch, int pairJoins, uint32_t tableCTAs, uint32_t *edge_out,
                             uint32_t *state_out, uint64_t *stats, int nthreads);

/* The bit join on the same phased schedule; outputs and stats as
 * oracle_join_bit plus [3] phases and [4] phases with two joins. */
int oracle_join_bit_phased(uint32_t ntip, uint32_t nbin, const uint32_t *words, const double *w,
                           int ancestralType, uint32_t maxBatch, int pairJoins, uint32_t tableCTAs,
                           uint32_t *edge_out, uint32_t *state_out, uint64_t *stats, int nthreads);

/* joinEdgeBitReverse.  words: ntip x nbin row-major bit rows.  w: nbin*32
 * doubles.  ancestralType 0 or 1 (any non-zero value selects rule 1). */
int oracle_join_bit(uint32_t ntip, uint32_t nbin, const uint32_t *words,
                    const double *w, int ancestralType, uint32_t *edge_out,
                    uint32_t *state_out, uint64_t *stats, int nthreads);

/* nodeKeepIndel / nodeKeepBit.  Writes retained node ids (in the order the
 * reference prints them) to out_nodes, count to *nout. */
int oracle_node_keep_indel(uint32_t nnodeRows, uint32_t ncol, const uint32_t *nodeState,
                           uint32_t nedge, const uint32_t *edge, uint32_t nRetain,
                           const uint32_t *outmat, uint32_t cutoff,
                           uint32_t *out_nodes, uint32_t *nout);
int oracle_node_keep_bit(uint32_t nnodeRows, uint32_t nbin, const uint32_t *nodeState,
                         uint32_t nedge, const uint32_t *edge, uint32_t nRetain,
                         const uint32_t *outmat, uint32_t cutoff,
                         uint32_t *out_nodes, uint32_t *nout);

/* radiusNeighbor.  bmat: word-plane-major (nrow words x ntip).  counts[ntip];
 * idx (nullable) receives the concatenated ascending lists. */
int oracle_radius_bit(uint32_t nrow, uint32_t ntip, const uint32_t *bmat,
                      const double *w, int32_t radius, uint32_t *counts,
                      uint32_t *idx, uint64_t idx_cap, uint64_t *total,
                      int nthreads);
/* radiusNeighborDNA.  raw: ntip x nbinRaw fasta2bin words (4 codes/word). */
int oracle_radius_dna(uint32_t ntip, uint32_t nbinRaw, const uint32_t *raw,
                      uint32_t radius, uint32_t *counts, uint32_t *idx,
                      uint64_t idx_cap, uint64_t *total, int nthreads);
/* tryRadius / tryRadiusDNA with given query indices. */
int oracle_try_radius_bit(uint32_t nrow, uint32_t ntip, const uint32_t *bmat,
                          const double *w, int32_t radius, uint32_t nrep,
                          const uint32_t *qidx, uint32_t *counts, int nthreads);
int oracle_try_radius_dna(uint32_t ntip, uint32_t nbinRaw, const uint32_t *raw,
                          uint32_t radius, uint32_t nrep, const uint32_t *qidx,
                          uint32_t *counts, int nthreads);

/* TransferDisStream. */
int oracle_transfer_dis(uint32_t nrow_y, uint32_t nrow_x, uint32_t ncol, uint32_t ntip,
                        const uint32_t *y, const uint32_t *x, uint32_t *ymin,
                        uint32_t *ysize, uint32_t *xmin, uint32_t *xsize,
                        int nthreads);

/* Parsimony change counts per edge.  edge: nedge x 2 (parent, child), 0-based,
 * tips 0..ntip-1, internal nodes ntip..ntip+nnode-1, rows in pre-order
 * (parents before children, as an ape edge matrix).
 * ancestralBitReverse (src/functions.cpp:3478-3542): mat ntip x nbin words;
 *   state_out, bistate_out nnode x nbin; len_out[nedge].
 * charAncestralEC (src/functions.cpp:3085-3150): mat ntip x nsite int32
 *   (-1 unknown); state_out nnode x nsite; len_out[nedge]. */
int oracle_ancestral_bit(uint32_t ntip, uint32_t nnode, uint32_t nbin, const uint32_t *mat,
                         uint32_t nedge, const uint32_t *edge, uint32_t *state_out,
                         uint32_t *bistate_out, uint32_t *len_out);
int oracle_ancestral_char(uint32_t ntip, uint32_t nnode, uint32_t nsite, const int32_t *mat,
                          uint32_t nedge, const uint32_t *edge, const uint32_t *tipSize,
                          float minSize, float minRatio, int32_t *state_out, uint32_t *len_out);

/* nodeDesBig (src/functions.cpp:1277-1366): rows_out gets, for the internal
 * children in reverse edge order, their tip bitsets ((nnode-1) x nbin u32,
 * nbin = (ntip-1)/32+1: the file body); sizes_out[nnode-1] the returned
 * sizes.  ORACLE_ERANGE where the reference runs out of its 8192 cache rows. */
int oracle_node_des(uint32_t ntip, uint32_t nnode, uint32_t nedge, const uint32_t *edge,
                    uint32_t *rows_out, int32_t *sizes_out);

/* tipMerge (cu/tipMerge.cu:130-461): counts[ntip] and the concatenated
 * ascending neighbour lists idx (the .nNeighbor body and .idx); member_out
 * gets the .member values.  Returns ORACLE_ERANGE when a list is longer than
 * 1048576 (the reference prints a message and writes nothing). */
int oracle_tip_merge(uint32_t ntip, const uint32_t *counts, const uint32_t *idx, double pShared,
                     int32_t *member_out);

/* approximateCompare2_AVX2 (src/functions.cpp:5450-5600): transfer-style
 * matching of the clades of a query tree (edge2) against those of a
 * reference tree (edge1, clade rows as nodeDesBig writes them: row k = node
 * ntip+nnode1-1-k).  Edges are 0-based (parent, child) pairs in cladewise
 * order, tips 0..ntip-1, root ntip.  ref2qry: nnode1 x 2 row-major (1-based
 * node of the query tree, distance), qry2ref: nnode2 x 3 row-major (1-based
 * node of the reference tree, distance, size).  Returns ORACLE_ERANGE where
 * the reference runs out of its cacheSize open rows. */
int oracle_approx_compare(uint32_t ntip, uint32_t nnode1, uint32_t nbin, const uint32_t *clade, uint32_t nedge1,
                          const uint32_t *edge1, uint32_t nedge2, const uint32_t *edge2, uint32_t nnode2,
                          uint32_t cacheSize, float threshold, int32_t *ref2qry, int32_t *qry2ref);

/* FP64 log-likelihoods (Felsenstein pruning) for branch-length checks at
 * full size.  edge: nedge x 2 (parent, child), tips 0..ntip-1, binary, one
 * root.  weights (nullable) per site.  HKY85 on fasta2bin nibbles;
 * irreversible edits on .tbmat codes with q: nsite x (K+1) allele
 * frequencies (column 0 unused). */
int oracle_loglik_hky85(uint32_t ntip, uint32_t nedge, const uint32_t *edge, const double *t, uint32_t nsite,
                        const uint32_t *codes, const double *weights, double kappa, const double *pi, double *ll,
                        int nthreads);
int oracle_loglik_irreversible(uint32_t ntip, uint32_t nedge, const uint32_t *edge, const double *t, uint32_t nsite,
                               const uint32_t *codes, const double *weights, uint32_t K, const double *q,
                               double rate, double *ll, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
