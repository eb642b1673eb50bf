/*
 * casphy.h -- C ABI of libcasphy.so, the B200 (sm_100a) implementation of
 * CasPhy's tree-building hot path.
 *
 * Every entry point takes plain host pointers and sizes (the *_dev variants
 * take device pointers and an optional cudaStream_t passed as void*), returns
 * an int status (0 = CASPHY_OK) and never exits the process.  Outputs are the
 * exact bytes the corresponding reference executable writes (minus the file
 * headers, which the drop-in executables add).  Cited paths are relative to
 * the CasPhy source tree.
 */
#ifndef CASPHY_H
#define CASPHY_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CASPHY_ABI_VERSION 2

#define CASPHY_OK 0
#define CASPHY_EINVAL 1     /* bad argument (size, weight, code out of range) */
#define CASPHY_ERANGE 2     /* a value exceeds a documented limit */
#define CASPHY_ENOMEM 3     /* device or host allocation failed */
#define CASPHY_ECUDA 4      /* CUDA runtime error (see casphy_last_error) */
#define CASPHY_ETIMEOUT 5   /* a bounded device-side wait gave up */
#define CASPHY_EIO 6        /* file missing / truncated (drop-in executables) */
#define CASPHY_ENODEV 7     /* no CUDA device */
#define CASPHY_EINTERNAL 9  /* invariant violated (bug) */

int casphy_abi_version(void);
const char *casphy_strerror(int status);
/* Text of the last CUDA failure seen by this thread ("" if none). */
const char *casphy_last_error(void);
/* Number of visible CUDA devices (0 if none) and selection of the device the
 * calling thread's subsequent calls run on. */
int casphy_device_count(void);
int casphy_set_device(int device);

/* Statistics of one greedy join. */
typedef struct {
    uint64_t joins;              /* ntip - 1 */
    uint64_t stale_recomputes;   /* partner-already-joined rescans */
    uint64_t pair_scores;        /* (query, candidate) scores evaluated */
    uint64_t compactions;        /* slot-matrix compactions */
    uint64_t kernel_launches;    /* kernels launched by this call */
    uint32_t int_path;           /* 1: exact integer accumulation was used */
    uint32_t scan_path;          /* indel: 0 column-major codes, 1 allele bitsets */
    double init_scan_ms;         /* device time, initial all-pairs scan */
    double join_loop_ms;         /* device time, persistent join loop */
    double total_ms;             /* device time of the whole call */
    uint64_t alg_bytes_init;     /* algorithmic bytes of the initial scan */
    uint64_t alg_bytes_join;     /* algorithmic bytes of the join-loop scans */
    uint64_t phases;             /* grid-wide phases of the join loop */
    uint64_t refreshes;          /* republish phases (exhausted per-CTA lists) */
} casphy_join_stats;

/*
 * Greedy shared-mutation join of indel-coded cells.
 * Replaces the computation of `joinEdgeIndel <prefix> <wfile> <nState>
 * <minSize> <minRatio>` (cu/joinEdgeIndel.cu:244-578).
 *   codes     ntip x ncol u32, row-major: 0 missing, 1 unedited, >= 2 allele
 *             (the .tbmat body; R writes mat+1L, R/CasPhy_functions.R:610)
 *   weight    nState x ncol float64, weight of allele code c at site i is
 *             weight[(c-2)*ncol + i] (the .w file, R/CasPhy_functions.R:609)
 *   tipSize   ntip u32 (the .tipSize body)
 *   edge_out  (2*ntip-2) x 2 u32: the .edge2 body (pre-order relabelled,
 *             tips 0..ntip-1, root ntip)
 *   state_out max(ntip-1,1) x ncol u32: the .nodeState2 body (root first)
 * Weights must be finite and >= 0; codes must be <= nState+1 and < 65536.
 */
int casphy_join_indel(uint32_t ntip, uint32_t ncol, const uint32_t *codes,
                      uint32_t nState, const double *weight, const uint32_t *tipSize,
                      uint32_t minSize, float minRatio, uint32_t *edge_out,
                      uint32_t *state_out, casphy_join_stats *stats);

/* Same with device-resident codes / outputs (d_state_out may be NULL). */
int casphy_join_indel_dev(uint32_t ntip, uint32_t ncol, const uint32_t *d_codes,
                          uint32_t nState, const double *weight, const uint32_t *tipSize,
                          uint32_t minSize, float minRatio, uint32_t *edge_out,
                          uint32_t *d_state_out, casphy_join_stats *stats, void *stream);

/*
 * Greedy join of bit-coded cells.  Replaces `joinEdgeBitReverse <prefix>
 * <wfile> <ancestralType>` (cu/joinEdgeBitReverse.cu:285-615).
 *   words     ntip x nbin u32 bit rows (bit j of word k = site 32k+j; the
 *             .tbmat body)
 *   weight    nbin*32 float64 per-site weights (the .w file); >= 0, not NaN
 *   ancestralType 0 (updateAncestralKernel) or non-zero (updateAncestralKernel2)
 *   edge_out  (2*ntip-2) x 2 u32 (.edge2 body); state_out max(ntip-1,1) x nbin
 *             u32 (.nodeState2 body: seq & ~bistate, root first)
 */
int casphy_join_bit(uint32_t ntip, uint32_t nbin, const uint32_t *words,
                    const double *weight, int ancestralType, uint32_t *edge_out,
                    uint32_t *state_out, casphy_join_stats *stats);
/* Same with device-resident words / states. */
int casphy_join_bit_dev(uint32_t ntip, uint32_t nbin, const uint32_t *d_words,
                        const double *weight, int ancestralType, uint32_t *edge_out,
                        uint32_t *d_state_out, casphy_join_stats *stats, void *stream);

/*
 * nodeKeepIndel / nodeKeepBit (cu/nodeKeepIndel.cu:51-169,
 * cu/nodeKeepBit.cu:77-230).  nodeState: (ntip-1) x ncol u32 (the
 * .nodeState2 body; ncol = nbin words for the bit version), edge: nedge x 2
 * u32 (the .edge2 body), outmat: nRetain x ncol u32 (the .tboutmat body).
 * Writes the retained node ids in the order the reference prints them to
 * .retainNode (out_nodes must hold nedge entries) and their count.
 */
int casphy_node_keep_indel(uint32_t nnodeRows, uint32_t ncol, const uint32_t *nodeState,
                           uint32_t nedge, const uint32_t *edge, uint32_t nRetain,
                           const uint32_t *outmat, uint32_t cutoff, uint32_t *out_nodes,
                           uint32_t *nout);
int casphy_node_keep_bit(uint32_t nnodeRows, uint32_t nbin, const uint32_t *nodeState,
                         uint32_t nedge, const uint32_t *edge, uint32_t nRetain,
                         const uint32_t *outmat, uint32_t cutoff, uint32_t *out_nodes,
                         uint32_t *nout);

/*
 * radiusNeighbor (cu/radiusNeighbor.cu:162-470): bmat is the .bmat body,
 * word-plane-major (nrow words x ntip), weight the .w file (nrow*32 float64),
 * radius the integer argv value.  counts[ntip] receives the .nNeighbor body;
 * when idx is non-NULL and idx_cap >= the total, idx receives the .idx body
 * (for every row the ascending rows j with score >= radius).  *total gets the
 * list length either way.  Either call once with idx = NULL to size the
 * buffer, or pass a buffer of a guessed size: when the lists do not fit, the
 * call returns CASPHY_ERANGE with counts and *total filled (*total > idx_cap)
 * and a second call with a large enough buffer is needed.
 */
int casphy_radius_bit(uint32_t nrow, uint32_t ntip, const uint32_t *bmat, const double *weight,
                      int32_t radius, uint32_t *counts, uint32_t *idx, uint64_t idx_cap,
                      uint64_t *total);
/* radiusNeighborDNA (cu/radiusNeighborDNA.cu:111-380): raw is the fasta2bin
 * .bin body (ntip x nbinRaw u32, four 8-bit codes per word). */
int casphy_radius_dna(uint32_t ntip, uint32_t nbinRaw, const uint32_t *raw, uint32_t radius,
                      uint32_t *counts, uint32_t *idx, uint64_t idx_cap, uint64_t *total);
/* The same searches with the lists in a host buffer the library allocates
 * at their exact size once they are counted, so every search runs once
 * whatever its result size (the caller-buffer forms above need a second
 * search when the lists outgrow the buffer).  *idx_out receives the .idx body
 * (total entries), to be released with casphy_free; on failure it is NULL. */
int casphy_radius_bit_lists(uint32_t nrow, uint32_t ntip, const uint32_t *bmat, const double *weight,
                            int32_t radius, uint32_t *counts, uint32_t **idx_out, uint64_t *total);
int casphy_radius_dna_lists(uint32_t ntip, uint32_t nbinRaw, const uint32_t *raw, uint32_t radius,
                            uint32_t *counts, uint32_t **idx_out, uint64_t *total);
void casphy_free(void *p);
/* The lists of query rows [row_begin, row_end) only (counts has row_end -
 * row_begin entries, idx their concatenated lists): one GPU's share when the
 * rows are split over several GPUs. */
int casphy_radius_bit_rows(uint32_t nrow, uint32_t ntip, const uint32_t *bmat, const double *weight,
                           int32_t radius, uint32_t row_begin, uint32_t row_end, uint32_t *counts,
                           uint32_t *idx, uint64_t idx_cap, uint64_t *total);
int casphy_radius_dna_rows(uint32_t ntip, uint32_t nbinRaw, const uint32_t *raw, uint32_t radius,
                           uint32_t row_begin, uint32_t row_end, uint32_t *counts, uint32_t *idx,
                           uint64_t idx_cap, uint64_t *total);
/* tryRadius / tryRadiusDNA (cu/tryRadius.cu:52-189, cu/tryRadiusDNA.cu:76-178)
 * with the query rows given in qidx (the tools draw them with rand()). */
int casphy_try_radius_bit(uint32_t nrow, uint32_t ntip, const uint32_t *bmat, const double *weight,
                          int32_t radius, uint32_t nrep, const uint32_t *qidx, uint32_t *counts);
int casphy_try_radius_dna(uint32_t ntip, uint32_t nbinRaw, const uint32_t *raw, uint32_t radius,
                          uint32_t nrep, const uint32_t *qidx, uint32_t *counts);

/*
 * TransferDisStream (cu/TransferDisStream.cu:130-344): y and x are clade
 * bitset rows (nrow x ncol u32, the bodies of the two input files); outputs
 * are the value arrays of <out>_ymin.bin / <out>_xmin.bin (min transfer
 * distance and clade size per row).
 */
int casphy_transfer_dis(uint32_t nrow_y, uint32_t nrow_x, uint32_t ncol, uint32_t ntip,
                        const uint32_t *y, const uint32_t *x, uint32_t *ymin, uint32_t *ysize,
                        uint32_t *xmin, uint32_t *xsize);

/*
 * Bootstrap column resampling of a fasta2bin matrix (the gather of
 * cu/Felsenstein.cu:34-54): in is ntip x nbin u32 (4 byte codes per word),
 * idx holds nidx byte positions; out (ntip x ceil(nidx/4) u32) gets, in byte
 * j of word i of each row, the input byte at idx[4i+j] (0 for a position
 * past the row; bytes past nidx in the last word are 0).
 */
int casphy_resample_columns(uint32_t ntip, uint32_t nbin, const uint32_t *in, uint32_t nidx,
                            const uint32_t *idx, uint32_t *out);

/*
 * Felsenstein pruning and branch-length optimisation.  No counterpart in the
 * reference (its cu/Felsenstein.cu is the column resampler above and its
 * branch lengths are parsimony change counts, src/functions.cpp:3480-3542).
 * The tree is given as an .edge2 body: nedge = 2*ntip-2 rows (parent, child),
 * tips 0..ntip-1, internal nodes ntip..2*ntip-2, every internal node with two
 * children; brlen[e] is the length of edge row e.  tip_codes is ntip x nsite
 * u32: for HKY85 the fasta2bin nibble (bit 0 A, 1 T, 2 C, 3 G, 0 = missing),
 * for the irreversible edit model the .tbmat coding (0 missing, 1 unedited,
 * c >= 2 allele c-1).  site_weights may be NULL (all 1).
 */
#define CASPHY_MODEL_HKY85 0
#define CASPHY_MODEL_IRREVERSIBLE 1
#define CASPHY_GRAD_ADJOINT 0       /* one outside (pre-order) pass per gradient */
#define CASPHY_GRAD_CENTRAL_DIFF 1  /* per-edge central differences, 2 evaluations per edge */

typedef struct {
    uint32_t model;             /* CASPHY_MODEL_* */
    uint32_t nallele;           /* irreversible: alleles 1..nallele */
    double kappa;               /* HKY85 transition/transversion rate ratio */
    double pi[4];               /* HKY85 base frequencies, order A, T, C, G */
    double rate;                /* irreversible: edit rate per unit length */
    const double *allele_freq;  /* irreversible: nsite x (nallele+1), column 0
                                   unused; NULL = the tips' allele frequencies */
    uint64_t mem_budget;        /* device bytes for partials (0 = no limit);
                                   sites are processed in chunks that fit */
} casphy_felsenstein_model;

typedef struct {
    uint32_t iterations;        /* accepted L-BFGS steps */
    uint32_t evaluations;       /* likelihood evaluations (graph launches),
                                   including a speculated unit step that the
                                   accept then discards */
    uint32_t site_chunks;
    uint32_t levels_inside;     /* tree height (inside launches per chunk) */
    uint32_t levels_outside;    /* depth levels (outside launches per chunk) */
    uint32_t reserved;
    double loglik_start, loglik_end;
    double seconds;             /* device time of the whole optimisation */
    uint64_t launches_per_eval; /* kernels in one evaluation graph */
    double eval_seconds;        /* device time inside the evaluation graphs */
} casphy_blopt_stats;

/* log L (FP32 partials with per-site power-of-two scaling, FP64 site sums) and,
 * when grad is non-NULL, d log L / d brlen for every edge by the adjoint pass. */
int casphy_felsenstein_loglik(uint32_t ntip, uint32_t nedge, const uint32_t *edge,
                              const double *brlen, uint32_t nsite, const uint32_t *tip_codes,
                              const double *site_weights, const casphy_felsenstein_model *model,
                              double *loglik, double *grad);
/* L-BFGS over log branch lengths (FP64 step on the device) until the relative
 * change of log L is <= rel_tol in 5 consecutive steps, no descent step is
 * found, or max_iter steps; brlen is
 * updated in place (clamped to [1e-8, 10]). */
int casphy_felsenstein_optimize(uint32_t ntip, uint32_t nedge, const uint32_t *edge, double *brlen,
                                uint32_t nsite, const uint32_t *tip_codes, const double *site_weights,
                                const casphy_felsenstein_model *model, int gradient_mode,
                                uint32_t max_iter, double rel_tol, casphy_blopt_stats *stats);

/*
 * fasta2bin's column classification and encoding (cu/fasta2bin.cu:47-206):
 * seqs is the aligned sequences, nseq rows of len characters.  variable[len]
 * gets 1 for a variable column (some base count, ambiguity codes counting for
 * each of their bases, strictly between 0 and nseq); *nkeep_out the number
 * kept; bin_out (when non-NULL and bin_cap >= nseq*ceil(nkeep/4)) the .bin
 * body: per sequence the kept columns' 8-bit codes, four per u32, low byte
 * first.  Parsing the FASTA text stays with the caller (the fasta2bin drop-in).
 */
int casphy_fasta_encode(uint32_t nseq, uint32_t len, const char *seqs, uint8_t *variable,
                        uint32_t *nkeep_out, uint32_t *bin_out, uint64_t bin_cap);

/*
 * nodeDesBig (src/functions.cpp:1277-1366): the clade matrix phy2clade
 * writes for TransferDisStream (R/bootstrap_functions.R:1-32).  edge as for
 * the parsimony entry points; rows_out gets (nnode-1) x nbin u32 rows, nbin =
 * (ntip-1)/32+1: the tip bitset of every internal child, in reverse edge
 * order (the file body after its {nnode-1, nbin} header); sizes_out[nnode-1]
 * gets the sizes nodeDesBig returns (internal nodes 1..nnode-1, last first).
 * CASPHY_ERANGE where the reference runs out of its 8192 open rows.
 */
int casphy_node_des(uint32_t ntip, uint32_t nnode, uint32_t nedge, const uint32_t *edge,
                    uint32_t *rows_out, int32_t *sizes_out);

/*
 * approximateCompare2_AVX2 (src/functions.cpp:5450-5600) for many query
 * trees at once, as clade.support / cal.abs apply it over bootstrap trees
 * (R/bootstrap_functions.R:34-57, :190-202).  Reference tree: edge1 (0-based
 * (parent, child) pairs, tips 0..ntip-1, root ntip, nnode1 internal nodes)
 * and its clade rows as casphy_node_des writes them ((nnode1-1) x nbin).
 * Query tree t: edges2 + 2*edge_off[t], edge_off[t+1]-edge_off[t] edges in
 * cladewise order over the same tips, nnode2_t = nedges - ntip + 1 internal
 * nodes.  Outputs, the function's two matrices row by row: ref2qry[ntree *
 * nnode1 * 2] (1-based query node, XOR distance) and qry2ref[sum nnode2_t *
 * 3] (1-based reference node, distance, clade size), trees in order.
 * status[t] = CASPHY_ERANGE where the function runs out of its cache_size
 * open rows (it returns 0 to R then; that tree's rows are zero).
 */
int casphy_approx_compare(uint32_t ntip, uint32_t nnode1, const uint32_t *clade_rows, uint32_t nedge1,
                          const uint32_t *edge1, uint32_t ntree, const uint64_t *edge_off, const uint32_t *edges2,
                          uint32_t cache_size, float threshold, int32_t *ref2qry, int32_t *qry2ref,
                          int32_t *status);

/*
 * cal.abs (R/bootstrap_functions.R:190-219): transfer support of every
 * internal node of the reference tree (edge1, cladewise) over ntree query
 * trees (as above): the fraction of trees whose approximateCompare2_AVX2
 * distance (run at threshold + 0.05) over the node's size is at most
 * threshold.  support[nnode1] and node_size[nnode1] are the two columns of
 * its result (node order, root first).  CASPHY_ERANGE with "Run out of
 * cache!" where nodeDesBig or the comparison runs out of its 8192 rows.
 */
int casphy_cal_abs(uint32_t ntip, uint32_t nedge1, const uint32_t *edge1, uint32_t ntree, const uint64_t *edge_off,
                   const uint32_t *edges2, double threshold, double *support, int32_t *node_size);

/*
 * tipMerge (cu/tipMerge.cu:130-461): categories of tips whose neighbour lists
 * overlap.  counts[ntip] and idx (the concatenated ascending lists) are the
 * .nNeighbor body and the .idx file of radiusNeighbor(DNA); member[ntip]
 * receives the .member values.  A list longer than 1048576 entries gives
 * CASPHY_ERANGE with the reference's message in casphy_last_error() (the
 * reference then writes no .member file).
 */
int casphy_tip_merge(uint32_t ntip, const uint32_t *counts, const uint32_t *idx, double pShared,
                     int32_t *member);

/*
 * Parsimony change counts per edge, the reference's branch lengths
 * (collapse.infoless / cal.nevo, R/CasPhy_functions.R:804-845).
 *   edge      nedge x 2 u32 (parent, child), 0-based: tips 0..ntip-1, internal
 *             nodes ntip..ntip+nnode-1; rows in pre-order (a node's parent edge
 *             before its own edges, as an ape cladewise edge matrix or .edge2)
 *   edge_len  nedge u32: changes on each edge row
 * casphy_ancestral_bit replaces ancestralBitReverse (src/functions.cpp:
 * 3478-3542): mat is ntip x nbin u32 bit rows, the root must be node ntip,
 * state_out (optional) nnode x nbin gets the resolved node states.
 * casphy_ancestral_char replaces charAncestralEC (src/functions.cpp:
 * 3085-3150): mat is ntip x nsite int32 (-1 unknown), tipSize[ntip] and the
 * minSize / minRatio rule as there; state_out (optional) nnode x nsite.
 */
int casphy_ancestral_bit(uint32_t ntip, uint32_t nnode, uint32_t nbin, const uint32_t *mat,
                         uint32_t nedge, const uint32_t *edge, uint32_t *state_out, uint32_t *edge_len);
int casphy_ancestral_char(uint32_t ntip, uint32_t nnode, uint32_t nsite, const int32_t *mat,
                          uint32_t nedge, const uint32_t *edge, const uint32_t *tipSize, float minSize,
                          float minRatio, int32_t *state_out, uint32_t *edge_len);

/*
 * Batched bootstrap of the bit join with transfer support.  Replaces running
 * joinEdgeBitReverse, the clade writer and TransferDisStream once per
 * replicate (vignettes/CasPhy.Rmd:255-291, R/bootstrap_functions.R:190-219).
 *   words        ntip x nbin u32, the full matrix (the .tbmat body)
 *   full_edge    (2*ntip-2) x 2 u32, the .edge2 body of the full-data tree
 *   replicate r  cells rep_cells[rep_offsets[r] .. rep_offsets[r+1]) (distinct
 *                full-matrix rows, in the order they become the replicate's
 *                tips 0..n_r-1) and integer site weights rep_weights[r*nbin*32
 *                ..] (column multiplicities of the resample)
 *   support      per clade of the full tree (its internal nodes except the
 *                root, in increasing node id): the number of replicates with
 *                ysize > 0 and ymin <= threshold * ysize
 *   ymin, ysize  optional, nrep x nclade: TransferDisStream's _ymin.bin values
 *                for the full-tree clades restricted to the replicate's cells
 *                against the replicate tree's clades (ntip = n_r)
 *   rep_raw_edges optional: per replicate, 2*(n_r-1) raw join edges (parent,
 *                child) in join order over the replicate's tip ids
 * Each replicate tree is the tree joinEdgeBitReverse builds from its rows and
 * weights (the same engine as casphy_join_bit).  The CTAs joining each
 * replicate come from a cost model refitted after every call on the device;
 * the environment variable CASPHY_BS_GROUP=g fixes g of them (at most 8) for
 * every replicate of 512 cells or more instead.
 */
typedef struct {
    uint32_t nrep, nclade;
    double prep_ms, join_ms, transfer_ms, total_ms;  /* device times */
    uint64_t kernel_launches;
    uint64_t join_phases;                            /* summed over replicates */
    uint32_t max_ctas_per_rep;                       /* CTAs the largest replicate's join used */
    uint32_t tuned;                                  /* 1 when the split came from measured costs */
    double join_longest_ms;                          /* longest single replicate join */
    double join_busy_ms;                             /* replicate joins summed (CTA-time) */
    double cost_alpha_us, cost_beta_us, cost_gamma_us;  /* per-phase cost model after this call */
    uint32_t graph;                                  /* 1 when the pass ran as one captured CUDA graph */
    uint32_t reserved;
} casphy_bootstrap_stats;

int casphy_bootstrap_bit(uint32_t ntip, uint32_t nbin, const uint32_t *words, const uint32_t *full_edge,
                         uint32_t nrep, const uint32_t *rep_offsets, const uint32_t *rep_cells,
                         const double *rep_weights, int ancestralType, double threshold,
                         uint32_t *support, uint32_t *ymin, uint32_t *ysize, uint32_t *rep_raw_edges,
                         casphy_bootstrap_stats *stats);

/*
 * Zero-allocation variant of casphy_join_indel_dev.  It has no counterpart
 * in the reference; it exists for callers that must not allocate device
 * memory during the call -- e.g. a framework that has already reserved the
 * GPU's memory for its own pool, or a latency-critical loop that cannot take
 * the device-wide synchronisation of cudaMalloc/cudaFree.  It never calls
 * cudaMalloc/cudaFree (or any allocating routine): inputs and outputs are the
 * caller's buffers and all working memory comes from one 64 MiB scratch
 * array compiled into libcasphy.so, held by every GPU that loads the library
 * until the process exits.
 *   d_codes      device, ntip x ncol u32 (as casphy_join_indel)
 *   weight       host, nState x ncol float64; tipSize host, ntip u32
 *   d_edge_out   device, (2*ntip-2) x 2 u32  (the .edge2 body)
 *   d_state_out  device, (ntip-1) x ncol u32 (the .nodeState2 body)
 * Needs ntip >= 2.  Sizes whose working set exceeds the 64 MiB scratch
 * (roughly ntip*ncol*14 bytes plus per-site tables) are rejected with
 * CASPHY_ERANGE and a message in casphy_last_error().  The CUDA runtime
 * reserves the scratch array on a device when it loads the library's device
 * code there: at context creation with CUDA_MODULE_LOADING=EAGER, otherwise
 * at the first indel join on that device (this call or casphy_join_indel*).
 * A caller that gives the rest of the GPU to its own pool should make one
 * call, or set CUDA_MODULE_LOADING=EAGER, before doing so; later calls change
 * no device allocation.  The first call on a device also looks up the
 * scratch address for that device, so make that first call before any stream
 * capture.  All calls on a device share the scratch and overwrite it: calls
 * whose GPU work overlaps race, so the library serialises them per device
 * and each call, on success and on error, returns only when its work on
 * `stream` has finished.  This variant uses the column-major u16 code scan
 * (not the allele-bitset scan) and relabels the tree in one device thread,
 * which suits its small sizes.
 */
int casphy_join_indel_noalloc(uint32_t ntip, uint32_t ncol, const uint32_t *d_codes,
                              uint32_t nState, const double *weight, const uint32_t *tipSize,
                              uint32_t minSize, float minRatio, uint32_t *d_edge_out,
                              uint32_t *d_state_out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* CASPHY_H */
